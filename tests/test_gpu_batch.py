"""Batched multi-view rendering against single-view rendering: every view
of a batch (depth cascades, main view, cubemap faces) is bit-identical to
the same view rendered alone through drawAll / shadowMap."""
import numpy as np
import pytest

from axi_visualizer_b200 import scenes as S

pytestmark = pytest.mark.gpu


def single(R, view, casc):
    R.set_view(view)
    R.draw.clearZBuffer()
    R.draw.drawAll(R.shaders, shadowIds=casc)
    r, g, b, db = [x.copy() for x in R.draw.getFrame()]
    return r, g, b, db, R.draw.getIDs()[0]


@pytest.mark.parametrize("seed", [3, 1])
def test_batch_views_equal_single_views(seed):
    from axi_visualizer_b200.batch import Batch, cube_faces, scene_batch_views
    from axi_visualizer_b200.ops import SceneRenderer
    sc = S.scene_small(seed=seed, flags=S.MIP | S.SHADOW)
    main = S.default_view(320, 240, pos=(3, 2, -8))
    R = SceneRenderer(sc, 320, 240)
    descs = scene_batch_views(sc, main, faces_at=(0.0, 3.0, -6.0), face_side=64)
    B = Batch(R.draw, descs)
    flags = [g.flags for g in sc.groups]
    aidx = [g.alpha_index for g in sc.groups]
    for rep in range(2):                       # the second render replays the graph
        B.render(flags, aidx)
        R.shadow_pass()
        for k in range(len(sc.shadows)):
            assert np.array_equal(B.frame(k).view(np.uint32), R.draw.getSHM(k).view(np.uint32))
        casc = list(range(len(sc.shadows)))
        nd = len(sc.shadows)
        got = B.frame(nd)
        want = single(R, main, casc)
        for a, b in zip(got, want[:4]):
            assert np.array_equal(a.view(np.uint16 if a.dtype == np.uint16 else np.uint32),
                                  b.view(np.uint16 if b.dtype == np.uint16 else np.uint32))
        assert np.array_equal(B.ids(nd)[0], want[4])
        for j, fv in enumerate(cube_faces((0.0, 3.0, -6.0), 64)):
            Rf = SceneRenderer(sc, 64, 64)
            Rf.shadow_pass()
            got = B.frame(nd + 1 + j)
            want = single(Rf, fv, casc)
            assert np.array_equal(got[3].view(np.uint32), want[3].view(np.uint32))
            assert np.array_equal(got[0], want[0])
    st = B.stats()
    assert st["renders"] == 2 and st["grid"] > 0


def test_phased_mode_equals_persistent_mode():
    """The phased form (one kernel per phase in the graph, alpha-tested work
    on a parallel branch) gives the same bits as the persistent kernel, for
    every view, over several renders and chunk sizes."""
    from axi_visualizer_b200.batch import PERSISTENT, PHASED, Batch, scene_batch_views
    from axi_visualizer_b200.ops import SceneRenderer
    sc = S.scene_small(seed=4, flags=S.MIP | S.SHADOW, nquads=80)
    main = S.default_view(320, 240, pos=(3, 2, -8))
    R = SceneRenderer(sc, 320, 240)
    descs = scene_batch_views(sc, main, faces_at=(0.0, 3.0, -6.0), face_side=96)
    B = Batch(R.draw, descs)
    flags = [g.flags for g in sc.groups]
    aidx = [g.alpha_index for g in sc.groups]

    def all_views():
        out = []
        for k, d in enumerate(descs):
            f = B.frame(k)
            out.append([x.copy() for x in (f if isinstance(f, tuple) else (f,))])
            if d.kind == 0:
                out.append([B.ids(k)[0]])
        return out

    B.render(flags, aidx)
    want = all_views()
    for mode, chunk in ((PHASED, 16), (PHASED, 8), (PERSISTENT, 32), (PHASED, 32)):
        B.set_mode(mode)
        B.set_tuning(2, chunk)
        for _ in range(2):
            B.render(flags, aidx)
        got = all_views()
        for a, b in zip(got, want):
            for x, y in zip(a, b):
                assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), (mode, chunk)
    assert B.stats()["graph"]
