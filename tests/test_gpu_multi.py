"""The 4-way blend terrain material (av_draw_multi.c; F_MULTI) on the device
against the oracle, at the parity bars of test_gpu_parity; the batched
launch of the same views against the plain one; the material's argument
checks."""
import numpy as np
import pytest

import oracle as O
from axi_visualizer_b200 import scenes as S
from axi_visualizer_b200._lib import AxrError

from test_gpu_parity import check_frame, render_both

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [9, 10])
@pytest.mark.parametrize("pos", [(0, 30, -40), (5, 20, -20), (-10, 8, -12)])
def test_multi_scene_parity(seed, pos):
    sc = S.scene_multi(seed=seed)
    view = S.default_view(192, 144, pos=pos, target=(0, 12, 0))
    fr, smaps, got, R = render_both(sc, view)
    check_frame(fr, smaps, got, R)
    terrain = (fr.tri_id >= 0) & (fr.tri_id < sc.groups[0].ntris)
    assert terrain.sum() > 1000
    # the blend is exact on this path: every u16 colour value equals the oracle's
    r, g, b = got[:3]
    assert np.array_equal(r[terrain], fr.ro[terrain]) and np.array_equal(g[terrain], fr.go[terrain])
    assert np.array_equal(b[terrain], fr.bo[terrain])


def test_multi_scene_batched_equals_plain():
    from axi_visualizer_b200.batch import Batch, scene_batch_views
    sc = S.scene_multi(seed=9)
    view = S.default_view(192, 144, pos=(5, 20, -20), target=(0, 12, 0))
    fr, smaps, got, R = render_both(sc, view)
    B = Batch(R.draw, scene_batch_views(sc, view, faces_at=(0, 14, 0), face_side=128))
    B.render([g.flags for g in sc.groups], [g.alpha_index for g in sc.groups])
    nd = len(sc.shadows)
    br, bg, bb, bdb = B.frame(nd)
    r, g, b, db = got[:4]
    assert np.array_equal(bdb.view(np.uint32), db.view(np.uint32))
    assert np.array_equal(br, r) and np.array_equal(bg, g) and np.array_equal(bb, b)


def test_multi_material_checks():
    from axi_visualizer_b200.ops import SceneRenderer
    sc = S.scene_multi(seed=9)
    R = SceneRenderer(sc, 64, 48)
    R.set_view(S.default_view(64, 48, pos=(0, 30, -40), target=(0, 12, 0)))
    d = R.draw
    # the blend needs three groups after it
    shaders = list(R.shaders)
    shaders[3] = "multi"
    with pytest.raises(AxrError):
        d.drawAll(shaders, shadowIds=[0, 1])
    # and a single-level texture (group 4 has a mip chain)
    shaders = list(R.shaders)
    shaders[4] = "multi mip"
    with pytest.raises(AxrError):
        d.drawAll(shaders, shadowIds=[0, 1])
    # the refused calls left the handle usable
    d.drawAll(R.shaders, shadowIds=[0, 1])
    d.sync()
