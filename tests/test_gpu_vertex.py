"""The vertex stage on the device (CLDraw.rotate / transform / translate /
vertLight through the C ABI) against the oracle and the reference's golden
vectors: vertex arrays bit-exact, and the frames rendered from them at the
parity bars of test_gpu_parity (shadow maps, depth, ids, coverage exact)."""
import os
import sys

import numpy as np
import pytest

import oracle as O
from axi_visualizer_b200 import scenes as S
from axi_visualizer_b200._lib import AxrError

from test_gpu_parity import check_frame

GOLD = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLD)
import make_golden as MG  # noqa: E402

pytestmark = pytest.mark.gpu


def same(a, b):
    return a.shape == b.shape and np.array_equal(np.asarray(a, np.float32).view(np.uint32),
                                                 np.asarray(b, np.float32).view(np.uint32))


def renderer(sc, w, h):
    from axi_visualizer_b200.ops import SceneRenderer
    return SceneRenderer(sc, w, h)


def test_vertex_stage_golden():
    """The reference's vert.c run on the fixture's operations: the device
    arrays equal its output bit for bit, and so does the frame."""
    gold = np.load(os.path.join(GOLD, "ref_vertex.npz"))
    seed, (w, h, pos), ops, L = MG.vertex_ops()
    sc = S.scene_small(seed=seed, flags=0, with_alpha=True)
    R = renderer(sc, w, h)
    d = R.draw
    d.ambLight = np.float32(L["amb"])
    for kind, g, a, b, args in ops:
        if kind == "rotate":
            d.rotate(args[0], args[1], args[2], a, b, g)
        else:
            d.translate(args[0], a, b, g)
    d.vertLight(L["mask"], L["dir_int"], L["dir_dir"], L["point_int"], L["point_pos"], L["spot_int"],
                L["spot_dir"], L["spot_pos"])
    for g in range(len(sc.groups)):
        xyz, vn, li = d.getVertices(g)
        assert same(xyz, gold[f"g{g}_xyz"]), g
        assert same(vn, gold[f"g{g}_vn"]), g
        assert same(li, gold[f"g{g}_li"]), g
        sc.groups[g].xyz[...] = xyz; sc.groups[g].vn[...] = vn; sc.groups[g].li[...] = li
    view = S.default_view(w, h, pos=pos)
    R.frame(view)
    got = [x.copy() for x in d.getFrame()] + list(d.getIDs()) + [[d.getSHM(k) for k in range(len(sc.shadows))]]
    fr, smaps = O.render(sc, view)
    check_frame(fr, smaps, got)


@pytest.mark.parametrize("seed", [0, 5])
def test_vertex_stage_random_against_oracle(seed):
    """Random sub-ranges (unaligned starts and ends, empty, single vertex,
    whole group), rotations about random origins, translations, and light
    sets of every kind, on the composed shader's scene (mip, shadow, alpha)."""
    rng = np.random.default_rng(seed)
    sc = S.scene_small(seed=seed)
    w, h = 192, 144
    R = renderer(sc, w, h)
    d = R.draw
    ranges = [(0, None), (1, 2), (5, 5), (3, 4099), (4, 4096), (7, 8)]
    for step in range(12):
        g = int(rng.integers(0, len(sc.groups)))
        nv = sc.groups[g].ntris * 3
        a, b = ranges[step % len(ranges)] if step < len(ranges) else (int(rng.integers(0, nv)), None)
        a = min(a, nv)
        b = None if b is None else min(b, nv)
        end = nv if b is None else b
        G = sc.groups[g]
        if step % 3 != 2:
            old = MG.rot_mat(*rng.uniform(-3, 3, 3)); new = MG.rot_mat(*rng.uniform(-3, 3, 3))
            o = rng.uniform(-4, 4, 3)
            (d.rotate if step % 2 else d.transform)(old, new, o, a, b, g)
            O.transform(G.xyz, G.vn, old, new, o, a, end)
        else:
            c = rng.uniform(-2, 2, 3)
            d.translate(c, a, b, g)
            O.translate(G.xyz, c, a, end)
    lights = dict(pointI=rng.uniform(0, 3, (6, 3)), pointP=rng.uniform(-8, 8, (6, 3)),
                  spotI=rng.uniform(0, 3, (9, 3)), spotD=rng.standard_normal((9, 3)),
                  spotP=rng.uniform(-8, 8, (9, 3)))
    di, dd = rng.uniform(0, 2, (3, 3)), rng.standard_normal((3, 3))
    mask = [1] * len(sc.groups)
    d.vertLight(mask, di, dd, **lights)
    for g, G in enumerate(sc.groups):
        xyz, vn, li = d.getVertices(g)
        assert same(xyz, G.xyz) and same(vn, G.vn), g
        want = O.vert_light(G.xyz, G.vn, di, dd, d.ambLight, lights["pointI"], lights["pointP"], lights["spotI"],
                            lights["spotD"], lights["spotP"])
        assert same(li, want), g
        G.li[...] = want
    # None keeps the point and spot lights, 1 clears them
    d.vertLight([1, 0, 0], di, dd)
    assert same(d.getVertices(0)[2], sc.groups[0].li)
    d.vertLight([1, 0, 0], di, dd, 1, None, 1)
    want = O.vert_light(sc.groups[0].xyz, sc.groups[0].vn, di, dd, d.ambLight)
    assert same(d.getVertices(0)[2], want)
    sc.groups[0].li[...] = want
    view = S.default_view(w, h, pos=(2, 6, -18))
    R.frame(view)
    got = [x.copy() for x in d.getFrame()] + list(d.getIDs()) + [[d.getSHM(k) for k in range(len(sc.shadows))]]
    fr, smaps = O.render(sc, view)
    check_frame(fr, smaps, got)


def test_rotation_between_queued_shadow_passes():
    """shadowMap, rotate, shadowMap queued without a host wait: the second
    pass sees the rotated casters (the rotation waits for the first pass to
    finish reading, the second pass for the rotation)."""
    sc = S.scene_small(seed=2)
    R = renderer(sc, 64, 48)
    d = R.draw
    cast = [g.cast for g in sc.groups]
    old, new = np.eye(3), MG.rot_mat(0.2, 0.9, -0.3)
    ref0 = O.new_shadow_map(sc.shadows[0].dim)
    O.shadow_map(sc, 0, ref0)
    for rep in range(3):
        d.clearShadowMap(0)
        d.shadowMap(0, cast, R.shaders, sc.bias)
        d.rotate(old, new, (0.5, 0, 0.5), 0, None, 1)
        d.clearShadowMap(1)
        d.shadowMap(1, cast, R.shaders, sc.bias)
        G = sc.groups[1]
        O.transform(G.xyz, G.vn, old, new, (0.5, 0, 0.5), 0, G.ntris * 3)
        ref1 = O.new_shadow_map(sc.shadows[1].dim)
        O.shadow_map(sc, 1, ref1)
        assert np.array_equal(d.getSHM(1).view(np.uint32), ref1.view(np.uint32)), rep
        if rep == 0:
            assert np.array_equal(d.getSHM(0).view(np.uint32), ref0.view(np.uint32))


def test_vertex_stage_errors():
    sc = S.scene_small(seed=1)
    R = renderer(sc, 32, 32)
    d = R.draw
    nv = sc.groups[0].ntris * 3
    with pytest.raises(AxrError):
        d.rotate(np.eye(3), np.eye(3), (0, 0, 0), 0, nv + 1, 0)
    with pytest.raises(AxrError):
        d.translate((1, 0, 0), 5, 4, 0)
    with pytest.raises(AxrError):
        d.translate((1, 0, 0), 0, None, len(sc.groups))
    with pytest.raises(AxrError):
        d.vertLight([1] * len(sc.groups), np.ones((128, 3)), np.ones((128, 3)))
    with pytest.raises(ValueError):
        d.vertLight([1] * len(sc.groups), np.ones((2, 3)), np.ones((2, 3)), np.ones((2, 3)), np.ones((3, 3)))
    # nothing was changed by the refused calls
    xyz, vn, _ = d.getVertices(0)
    assert same(xyz, sc.groups[0].xyz) and same(vn, sc.groups[0].vn)


def test_copy_to_between_queued_shadow_passes():
    """shadowMap, copyTo, shadowMap: the second pass sees the copied
    geometry, and the first pass's map is the one of the old geometry."""
    sc = S.scene_small(seed=4)
    R = renderer(sc, 64, 48)
    d = R.draw
    cast = [g.cast for g in sc.groups]
    ref0 = O.new_shadow_map(sc.shadows[0].dim)
    O.shadow_map(sc, 0, ref0)
    G = sc.groups[1]
    moved = G.xyz.copy()
    moved[:, 1] += 1.5
    d.clearShadowMap(0)
    d.shadowMap(0, cast, R.shaders, sc.bias)
    d.copyTo(1, moved, G.vn, 0)
    d.clearShadowMap(1)
    d.shadowMap(1, cast, R.shaders, sc.bias)
    G.xyz[...] = moved
    ref1 = O.new_shadow_map(sc.shadows[1].dim)
    O.shadow_map(sc, 1, ref1)
    assert np.array_equal(d.getSHM(0).view(np.uint32), ref0.view(np.uint32))
    assert np.array_equal(d.getSHM(1).view(np.uint32), ref1.view(np.uint32))


def test_batched_render_after_rotation_equals_plain():
    """A rotation queued before a batched render: the batch (its captured
    graph) draws the rotated geometry, the same as the plain path and the
    oracle.  The batched main view is cleared to the plain frame's initial
    colour (1, 1, 1): an uncleared view keeps, where nothing covers it now,
    what its previous render drew there."""
    from axi_visualizer_b200.batch import Batch, depth, shaded
    sc = S.scene_small(seed=6)
    view = S.default_view(128, 96, pos=(3, 6, -16))
    R = renderer(sc, 128, 96)
    d = R.draw
    descs = [depth(c, sc.bias) for c in sc.shadows] + [shaded(view, [0, 1], clear=(1, 1, 1))]
    B = Batch(d, descs)
    flags, aidx = [g.flags for g in sc.groups], [g.alpha_index for g in sc.groups]
    B.render(flags, aidx)                           # the graph is captured before the rotation
    d.rotate(np.eye(3), MG.rot_mat(0.1, 0.7, 0.0), (0, 0, 0), 0, None, 1)
    B.render(flags, aidx)
    nd = len(sc.shadows)
    bmaps = [B.frame(k).copy() for k in range(nd)]
    br, bg, bb, bdb = [x.copy() for x in B.frame(nd)]
    bid = B.ids(nd)[0].copy()
    R.frame(view)
    G = sc.groups[1]
    O.transform(G.xyz, G.vn, np.eye(3), MG.rot_mat(0.1, 0.7, 0.0), (0, 0, 0), 0, G.ntris * 3)
    fr, smaps = O.render(sc, view)
    got = [x.copy() for x in d.getFrame()] + list(d.getIDs()) + [[d.getSHM(k) for k in range(nd)]]
    check_frame(fr, smaps, got)                     # the plain path
    r, g, b, db = got[:4]
    for k in range(nd):
        assert np.array_equal(bmaps[k].view(np.uint32), smaps[k].view(np.uint32)), f"batched cascade {k}"
    assert np.array_equal(bdb.view(np.uint32), db.view(np.uint32))
    assert np.array_equal(bid, got[4])
    diff = (br != r) | (bg != g) | (bb != b)
    ys, xs = np.nonzero(diff)
    assert not diff.any(), (f"{diff.sum()} px differ, e.g. {list(zip(ys[:5], xs[:5]))}: batched "
                            f"{[int(br[y, x]) for y, x in zip(ys[:5], xs[:5])]} plain "
                            f"{[int(r[y, x]) for y, x in zip(ys[:5], xs[:5])]} oracle "
                            f"{[int(fr.ro[y, x]) for y, x in zip(ys[:5], xs[:5])]} ids "
                            f"{[int(got[4][y, x]) for y, x in zip(ys[:5], xs[:5])]}")
