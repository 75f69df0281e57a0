"""Failure detection on the GPU without a GPU fault: the persistent batch
kernel's grid barrier is made to wait for blocks that are never launched
(host-side injection); every waiting block gives up after a short bounded
poll, the render reports "grid barrier timed out", the context stays usable
and the next normal render is exact."""
import time

import numpy as np
import pytest

from axi_visualizer_b200 import scenes as S

pytestmark = pytest.mark.gpu


def test_stalled_grid_barrier_ends_with_an_error_and_the_batch_recovers():
    from axi_visualizer_b200._lib import AxrError
    from axi_visualizer_b200.batch import PERSISTENT, Batch, scene_batch_views
    from axi_visualizer_b200.ops import SceneRenderer
    sc = S.scene_small(seed=3, flags=S.MIP | S.SHADOW)
    view = S.default_view(160, 128, pos=(3, 2, -8))
    R = SceneRenderer(sc, 160, 128)
    B = Batch(R.draw, scene_batch_views(sc, view))
    B.set_mode(PERSISTENT)
    flags = [g.flags for g in sc.groups]
    aidx = [g.alpha_index for g in sc.groups]
    B.render(flags, aidx)
    nd = len(sc.shadows)
    want = [x.copy() for x in B.frame(nd)]

    B.inject_barrier_stall(1, 4096)              # one block that never arrives; give up after 4096 polls
    t0 = time.perf_counter()
    B.render(flags, aidx)
    with pytest.raises(AxrError, match="grid barrier timed out"):
        B.frame(nd)
    assert time.perf_counter() - t0 < 30         # bounded: no hang

    B.inject_barrier_stall(0, 1 << 26)           # back to normal
    B.render(flags, aidx)
    got = B.frame(nd)
    for a, w in zip(got, want):
        assert np.array_equal(a.view(np.uint8), w.view(np.uint8))
    R.frame(view)                                # the handle's own path is unaffected
    assert R.draw.getFrame()[3].shape == (128, 160)
