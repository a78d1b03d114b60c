"""Inner faces of multi-block meshes on the CPU: registration of the mesh's
inner-interface records (InnerFace::register_boundary, reference
src/Mesh.cpp:39-172) and the oracle's inner_communication (reference
src/DataCommunication.cu:36-102).

* The library's cfk_register_inner_face and the oracle's restatement give the
  same face description, field for field, for records with every normal
  axis and side, reversed and permuted tangential axes, in 2-D and 3-D.
* After one communication the ghost nodes hold exactly the target nodes that
  the record's meaning names (same position along paired ranges, ghost depth
  g <-> target depth g), computed here independently with numpy, and the face
  nodes hold the two blocks' average.
* A block cut in two at node plane h steps like the whole block: inviscid air
  and the 2-D tube to 1e-14; mixtures to 1e-9, since the reference recomputes
  cv from bv at the communicated face nodes and for a mixture that goes
  through the temperature Newton iteration, whose residual is ~1e-11."""
import dataclasses
import itertools

import numpy as np
import pytest

import cases
import mechanism
import pyoracle
from multiblock import OracleBlocks, split_difference

import corefl_b200 as cfk


def _outflow_i(case):
    return dataclasses.replace(case, faces=[(f, d, 6 if f == 0 else lab) for f, d, lab in case.faces])


def _records_3d(m=(7, 6, 5), t=(6, 5, 7)):
    """Records of faces between blocks of extents m (this) and t (target):
    each normal axis and side on both blocks, either tangential axis marked
    (negated), paired with either target axis, in both senses."""
    out = []
    for face, side, tface, tside in itertools.product(range(3), (-1, 1), range(3), (-1, 1)):
        tang = [x for x in range(3) if x != face]
        ttang = [x for x in range(3) if x != tface]
        for a, p, flip_a, flip_b in itertools.product(tang, ttang, (False, True), (False, True)):
            b = next(x for x in tang if x != a)
            q = next(x for x in ttang if x != p)
            if m[a] != t[p] or m[b] != t[q]:
                continue
            src, tar = [0] * 6, [0] * 6
            src[2 * face] = src[2 * face + 1] = 1 if side < 0 else m[face]
            tar[2 * tface] = tar[2 * tface + 1] = 1 if tside < 0 else t[tface]
            src[2 * a], src[2 * a + 1] = -1, -m[a]      # the marked (first) tangential axis
            src[2 * b], src[2 * b + 1] = 1, m[b]
            rp = (t[p], 1) if flip_a else (1, t[p])
            rq = (t[q], 1) if flip_b else (1, t[q])
            tar[2 * p], tar[2 * p + 1] = -rp[0], -rp[1]
            tar[2 * q], tar[2 * q + 1] = rq
            out.append((src, tar))
    return out


def _fields(f):
    return {n: (list(getattr(f, n)) if hasattr(getattr(f, n), "__len__") else getattr(f, n)) for n, _ in f._fields_}


def test_registration_matches_library_and_hand_example():
    recs = _records_3d()
    assert len(recs) >= 40
    for src, tar in recs:
        a = pyoracle.register_inner_face(3, 3, src, tar, 2)
        b = cfk.register_inner_face(3, 3, src, tar, 2)
        assert bytes(a) == bytes(b), (src, tar)
    for src, tar in ([[7, 7, 1, 6, 1, 1], [1, 1, 6, 1, 1, 1]], [[1, 1, 1, 6, 1, 1], [1, 6, 4, 4, 1, 1]]):
        assert bytes(pyoracle.register_inner_face(2, 2, src, tar, 3)) == bytes(cfk.register_inner_face(2, 2, src, tar, 3))
    # i-max face of a 9-node block against the i-min face of its neighbour, ngg 3
    f = _fields(cfk.register_inner_face(3, 3, [9, 9, -1, -9, 1, 7], [1, 1, -1, -9, 1, 7], 2))
    assert f["range_start"] == [8, 0, 0] and f["range_end"] == [11, 8, 6] and f["n_point"] == [4, 9, 7]
    assert f["face"] == 0 and f["direction"] == 1 and f["target_block"] == 1 and f["target_direction"] == -1
    assert f["target_start"] == [0, 0, 0] and f["src_tar"] == [0, 1, 2] and f["target_loop_dir"] == [1, 1, 1]
    with pytest.raises(cfk.CfkError):
        cfk.register_inner_face(3, 3, [1, 9, 1, 9, 1, 7], [1, 1, -1, -9, 1, 7], 2)  # no normal axis
    with pytest.raises(cfk.CfkError):
        cfk.register_inner_face(3, 3, [9, 9, 1, 9, 1, 7], [1, 1, -1, -9, 1, 7], 2)  # no marked axis


def _expected_map(src, tar, m, t, g):
    """Node map of a record by its meaning: along the normal, ghost depth d
    behind this face <-> depth d inside the target; across it, the same
    position along the paired ranges (marked axis with marked axis).
    Returns {this 0-based (i, j, k): target 0-based (i, j, k)}."""
    def axes(r):
        normal = next(a for a in range(3) if r[2 * a] == r[2 * a + 1])
        tang = [a for a in range(3) if a != normal]
        marked = next(a for a in tang if r[2 * a] < 0)
        other = next(a for a in tang if a != marked)
        return normal, marked, other

    def nodes(r, a):
        s, e = abs(r[2 * a]) - 1, abs(r[2 * a + 1]) - 1
        return list(range(s, e + 1)) if s <= e else list(range(s, e - 1, -1))

    n, a1, a2 = axes(src)
    tn, t1, t2 = axes(tar)
    side = -1 if src[2 * n] == 1 else 1
    tside = -1 if tar[2 * tn] == 1 else 1
    out = {}
    for d in range(g + 1):
        for p, x1 in enumerate(nodes(src, a1)):
            for q, x2 in enumerate(nodes(src, a2)):
                me = [0, 0, 0]
                me[n] = (0 if side < 0 else m[n] - 1) + side * d
                me[a1], me[a2] = x1, x2
                tg = [0, 0, 0]
                tg[tn] = (0 if tside < 0 else t[tn] - 1) - tside * d
                tg[t1], tg[t2] = nodes(tar, t1)[p], nodes(tar, t2)[q]
                out[tuple(me)] = tuple(tg)
    return out


def _random_zone_case(m, g, seed):
    rng = np.random.default_rng(seed)
    base = cases.sine_wave(n=m[0], ny=m[1], nz=m[2], scheme=52, viscous=False)
    assert base.ngg == g
    bv = base.bv.copy()
    bv[0] = 1.0 + 0.1 * rng.random(bv.shape[1])
    bv[1:4] = rng.standard_normal((3, bv.shape[1]))
    bv[4] = 0.7 + 0.1 * rng.random(bv.shape[1])
    bv[5] = bv[4] / (bv[0] * cases.R_AIR)
    return dataclasses.replace(base, bv=bv, faces=[])


@pytest.mark.parametrize("k", range(0, 96, 7))
def test_communication_fills_the_record_map(k):
    m, t, g = (7, 6, 5), (6, 5, 7), 3
    recs = _records_3d(m, t)
    src, tar = recs[k % len(recs)]
    ca, cb = _random_zone_case(m, g, 1), _random_zone_case(t, g, 2)
    za, zb = pyoracle.OracleZone(ca), pyoracle.OracleZone(cb)
    za.call("orc_compute_cv_from_bv")
    a0, b0 = za["bv"].copy(), zb["bv"].copy()
    f = pyoracle.register_inner_face(3, g, src, tar, 2)
    za.inner_communication(zb, f)
    shape = lambda c: (6, c.mz + 2 * g, c.my + 2 * g, c.mx + 2 * g)
    A, B = za["bv"].reshape(shape(ca)), zb["bv"].reshape(shape(cb))
    A0, B0 = a0.reshape(shape(ca)), b0.reshape(shape(cb))
    emap = _expected_map(src, tar, m, t, g)
    assert len(emap) == np.prod(list(f.n_point))
    at = lambda X, n: X[:, n[2] + g, n[1] + g, n[0] + g]
    normal = f.face
    for me, tg in emap.items():
        if me[normal] == (0 if f.direction < 0 else m[normal] - 1):
            ave = 0.5 * (at(B0, tg) + at(A0, me))
            assert np.array_equal(at(A, me), ave) and np.array_equal(at(B, tg), ave)
        else:
            assert np.array_equal(at(A, me), at(B0, tg))
    # nothing else changed
    changed = np.argwhere(np.any(A != A0, axis=0))
    assert all(tuple(int(c) - g for c in reversed(n)) in emap for n in changed)


def test_wall_side_keeps_or_takes_values():
    """A face node at rest stays as it is; a moving node next to a target
    node at rest takes the target's values."""
    m, g = (7, 6, 5), 3
    ca, cb = _random_zone_case(m, g, 3), _random_zone_case(m, g, 4)
    src, tar = [7, 7, -1, -6, 1, 5], [1, 1, -1, -6, 1, 5]
    za, zb = pyoracle.OracleZone(ca), pyoracle.OracleZone(cb)
    sh = (6, m[2] + 2 * g, m[1] + 2 * g, m[0] + 2 * g)
    A, B = za["bv"].reshape(sh), zb["bv"].reshape(sh)
    A[1:4, g + 2, g + 1, g + m[0] - 1] = 0.0   # this side at rest
    B[1:4, g + 3, g + 4, g + 0] = 0.0          # target side at rest
    A0, B0 = A.copy(), B.copy()
    za.inner_communication(zb, pyoracle.register_inner_face(3, g, src, tar, 2))
    assert np.array_equal(A[:, g + 2, g + 1, g + m[0] - 1], A0[:, g + 2, g + 1, g + m[0] - 1])
    assert np.array_equal(B[:, g + 2, g + 1, g], B0[:, g + 2, g + 1, g])
    assert np.array_equal(A[:, g + 3, g + 4, g + m[0] - 1], B0[:, g + 3, g + 4, g])
    assert np.array_equal(B[:, g + 3, g + 4, g], B0[:, g + 3, g + 4, g])


def _split_vs_whole(whole, h, steps):
    A, B, links = cases.split_i(whole, h, periodic_i=False)
    oz = pyoracle.OracleZone(whole)
    oz.initialize()
    mb = OracleBlocks([A, B], links)
    mb.initialize()
    worst = 0.0
    for _ in range(steps):
        assert oz.step() == pytest.approx(mb.step(), rel=1e-13)
        worst = max(worst, split_difference(whole, oz["cv"], A, B, [mb.z[0]["cv"], mb.z[1]["cv"]], h))
    return worst


@pytest.mark.parametrize("scheme,h", [(52, 12), (72, 9)])
def test_split_block_steps_like_whole_block(scheme, h):
    whole = _outflow_i(cases.perturbed(cases.sine_wave(n=25, ny=11, nz=9, scheme=scheme, viscous=False), seed=3,
                                       amp=0.05))
    assert _split_vs_whole(whole, h, 4) <= 1e-14


@pytest.mark.parametrize("scheme,recon,h", [(52, 2, 30), (4, 2, 20)])
def test_split_2d_tube_steps_like_whole_tube(scheme, recon, h):
    assert _split_vs_whole(cases.sod(64, 9, scheme=scheme, reconstruction=recon), h, 4) <= 1e-14


def test_split_mixture_steps_like_whole_block():
    mech = mechanism.load("li2004")
    whole = _outflow_i(cases.perturbed(cases.mix_wave(mech, 15, ny=9, nz=7, scheme=52, viscous=False), seed=2,
                                       amp=1e-2))
    assert _split_vs_whole(whole, 7, 3) <= 1e-9


def test_periodic_split_stays_finite_and_consistent():
    """A periodic block cut in two with its periodic i faces turned into an
    inner face as well: after steps of the viscous wave the duplicated
    planes of the two blocks hold the same values."""
    whole = cases.perturbed(cases.sine_wave(n=25, ny=11, nz=9, scheme=72, viscous=True), seed=3, amp=0.02)
    A, B, links = cases.split_i(whole, 12)
    assert len(links) == 4
    mb = OracleBlocks([A, B], links)
    mb.initialize()
    for _ in range(3):
        mb.step()
    g = whole.ngg
    sh = lambda c: (c.param["n_var"], c.mz + 2 * g, c.my + 2 * g, c.mx + 2 * g)
    a, b = mb.z[0]["bv"].reshape((6,) + sh(A)[1:]), mb.z[1]["bv"].reshape((6,) + sh(B)[1:])
    inner = (slice(None), slice(g, g + whole.mz), slice(g, g + whole.my))
    assert np.all(np.isfinite(a)) and np.all(np.isfinite(b))
    assert np.array_equal(a[inner][..., g + A.mx - 1], b[inner][..., g])      # the cut
    assert np.array_equal(a[inner][..., g], b[inner][..., g + B.mx - 1])      # the periodic seam


def _inner_file(links, n_block):
    """The mesh's inner-interface file for `links` in the layout of the
    reference's reader: title, per-block face counts, title, record pairs."""
    lines = ["inner faces", " ".join(str(sum(1 for b, *_ in links if b == k)) for k in range(n_block)), "records"]
    for k in range(n_block):
        for b, src, tar, tb in links:
            if b == k:
                lines.append(" ".join(map(str, src + [0])))
                lines.append(" ".join(map(str, tar + [tb])))
    return "\n".join(lines) + "\n"


@pytest.mark.parametrize("periodic", [True, False])
def test_inner_interface_file_registers_like_the_records(tmp_path, periodic):
    whole = cases.sine_wave(n=25, ny=11, nz=9, scheme=52, viscous=False)
    if not periodic:
        whole = _outflow_i(whole)
    A, B, links = cases.split_i(whole, 12)
    path = tmp_path / "inner   0.txt"
    path.write_text(_inner_file(links, 2))
    per_block = cfk.read_inner_interface(path, 3, whole.ngg, 2)
    for k in range(2):
        want = [cfk.register_inner_face(3, whole.ngg, s, t, tb) for b, s, t, tb in links if b == k]
        assert [bytes(f) for f in per_block[k]] == [bytes(f) for f in want]
    assert len(per_block[0]) == (2 if periodic else 1)
    # the same file for the 2-D tube
    A2, B2, links2 = cases.split_i(cases.sod(64, 9, scheme=52), 30)
    (tmp_path / "inner2.txt").write_text(_inner_file(links2, 2))
    got = cfk.read_inner_interface(tmp_path / "inner2.txt", 2, 3, 2)
    assert bytes(got[1][0]) == bytes(cfk.register_inner_face(2, 3, links2[1][1], links2[1][2], links2[1][3]))


def test_inner_interface_file_errors(tmp_path):
    whole = cases.sine_wave(n=25, ny=11, nz=9, scheme=52, viscous=False)
    _, _, links = cases.split_i(whole, 12)
    text = _inner_file(links, 2)
    with pytest.raises(cfk.CfkError, match="-5: cannot open"):
        cfk.read_inner_interface(tmp_path / "missing.txt", 3, 3, 2)
    (tmp_path / "cut.txt").write_text("\n".join(text.splitlines()[:-1]) + "\n")
    with pytest.raises(cfk.CfkError, match="file ends inside block 1"):
        cfk.read_inner_interface(tmp_path / "cut.txt", 3, 3, 2)
    (tmp_path / "f.txt").write_text(text)
    with pytest.raises(cfk.CfkError, match="max_faces"):
        cfk.read_inner_interface(tmp_path / "f.txt", 3, 3, 2, max_faces=3)
    bad = text.replace("-1 -11 1 9", "1 11 1 9", 1)   # first record loses its marked axis
    (tmp_path / "bad.txt").write_text(bad)
    with pytest.raises(cfk.CfkError, match="cannot be decoded"):
        cfk.read_inner_interface(tmp_path / "bad.txt", 3, 3, 2)


def _outflow_axis(case, axis):
    return dataclasses.replace(case, faces=[(f, d, 6 if f == axis else lab) for f, d, lab in case.faces])


def _split_vs_whole_axis(whole, h, axis, steps):
    A, B, links = cases.split(whole, h, axis, periodic=False)
    oz = pyoracle.OracleZone(whole)
    oz.initialize()
    mb = OracleBlocks([A, B], links)
    mb.initialize()
    g = whole.ngg
    shp = lambda c: (-1, c.mz + 2 * g, c.my + 2 * g, c.mx + 2 * g)
    worst = 0.0
    for _ in range(steps):
        assert oz.step() == pytest.approx(mb.step(), rel=1e-13)
        W = oz["cv"].reshape(shp(whole))
        scale = np.abs(W).max(axis=(1, 2, 3))
        scale[1:4] = scale[1:4].max()
        for blk, lo in ((A, 0), (B, h)):
            arr = (mb.z[0] if blk is A else mb.z[1])["cv"].reshape(shp(blk))
            inner = arr[:, g:g + blk.mz, g:g + blk.my, g:g + blk.mx]
            sl = [slice(None), slice(g, g + whole.mz), slice(g, g + whole.my), slice(g, g + whole.mx)]
            sl[3 - axis] = slice(g + lo, g + lo + (blk.mx, blk.my, blk.mz)[axis])
            worst = max(worst, float((np.abs(inner - W[tuple(sl)]) / scale[:, None, None, None]).max()))
    return worst


@pytest.mark.parametrize("axis,h", [(1, 5), (2, 4)])
def test_block_cut_across_j_or_k_steps_like_whole_block(axis, h):
    """The cut across j (tangential axes i marked, k) and across k (i marked,
    j): registration and communication for the other normal axes, over
    whole RK3 steps."""
    whole = _outflow_axis(cases.perturbed(cases.sine_wave(n=13, ny=12, nz=10, scheme=52, viscous=False), seed=4,
                                          amp=0.05), axis)
    assert _split_vs_whole_axis(whole, h, axis, 3) <= 1e-14


def test_2d_tube_cut_across_j_steps_like_whole_tube():
    assert _split_vs_whole_axis(cases.sod(40, 12, scheme=52), 6, 1, 4) <= 1e-14
