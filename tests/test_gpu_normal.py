"""The normal-mapped materials on the GPU against the oracle.

av_draw_normmap.c (plain and metal), av_draw_normmap_alpha.c and
av_draw_normmap_mip.c on one raster (scenes.scene_normal: normal-mapped
terrain, metal icospheres, trilinear icospheres with a normal-map chain,
alpha-tested quads, two cascades).  The oracle's restatement of these
materials is pinned to the reference's own kernels (tests/test_oracle_pin.py).
Coverage, triangle ids, depth and the shadow maps bit-exact, colour within
1/255 after gamma (the frames reached here are identical u16 planes), and
the same view as one batched launch bit for bit.
"""
import numpy as np
import pytest

import oracle as O
from axi_visualizer_b200 import scenes as S

from test_gpu_parity import check_frame

pytestmark = pytest.mark.gpu

VIEWS = [(2, 6, -14), (-4, 9, -10), (0, 20, -2)]


@pytest.mark.parametrize("pos", VIEWS)
def test_normal_mapped_frame_equals_oracle(pos):
    from axi_visualizer_b200.ops import SceneRenderer
    sc = S.scene_normal(seed=6)
    view = S.default_view(192, 144, pos=pos)
    fr, smaps = O.render(sc, view)
    R = SceneRenderer(sc, view.w, view.h, device=0)
    R.frame(view)
    r, g, b, db = [x.copy() for x in R.draw.getFrame()]
    tid, cov = R.draw.getIDs()
    shm = [R.draw.getSHM(k) for k in range(len(sc.shadows))]
    exact, psnr = check_frame(fr, smaps, (r, g, b, db, tid, cov, shm))
    for gi in range(len(sc.groups)):
        base = sum(x.ntris for x in sc.groups[:gi])
        assert ((tid >= base) & (tid < base + sc.groups[gi].ntris)).any(), f"group {gi} is visible"
    assert exact == 1.0, f"u16 planes: exact fraction {exact}"


def test_normal_mapped_batch_equals_plain():
    from axi_visualizer_b200.batch import Batch, scene_batch_views
    from axi_visualizer_b200.ops import SceneRenderer
    sc = S.scene_normal(seed=13)
    view = S.default_view(192, 144, pos=VIEWS[0])
    R = SceneRenderer(sc, view.w, view.h, device=0)
    R.frame(view)
    want = [x.copy() for x in R.draw.getFrame()]
    B = Batch(R.draw, scene_batch_views(sc, view))
    B.render([gp.flags for gp in sc.groups], [gp.alpha_index for gp in sc.groups])
    got = B.frame(len(sc.shadows))
    for a, w in zip(got, want):
        assert np.array_equal(a.view(np.uint8), w.view(np.uint8))
