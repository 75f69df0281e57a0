"""Edge cases on the GPU: the CUDA path against the oracle on the
known-answer scenes, the tile-unit queue overflow fallback, masked and empty
groups, and the error behaviour of the API."""
import os

import numpy as np
import pytest

import kat
import oracle as O
from axi_visualizer_b200 import scenes as S

pytestmark = pytest.mark.gpu
SCENES, VIEW = kat.case_scenes()


def cuda_frame(sc, view, mask=None):
    from axi_visualizer_b200.ops import SceneRenderer
    R = SceneRenderer(sc, view.w, view.h)
    R.shadow_pass()
    R.set_view(view)
    R.draw.clearZBuffer()
    uses = any(g.flags & S.SHADOW for g in sc.groups)
    R.draw.drawAll(R.shaders, mask=mask, shadowIds=list(range(min(2, len(sc.shadows)))) if uses else [])
    r, g, b, db = [x.copy() for x in R.draw.getFrame()]
    tid, cov = R.draw.getIDs()
    return (r, g, b, db, tid, cov, [R.draw.getSHM(k) for k in range(len(sc.shadows))]), R


def oracle_frame(sc, view, mask=None):
    smaps = []
    for k, s in enumerate(sc.shadows):
        m = O.new_shadow_map(s.dim)
        O.shadow_map(sc, k, m)
        smaps.append(m)
    fr = O.Frame(view.w, view.h)
    O.clear_depth(fr.db)
    O.draw_all(sc, view, fr, [], mask=mask)
    return fr, smaps


def assert_same(fr, smaps, got):
    r, g, b, db, tid, cov, shm = got
    for k, m in enumerate(smaps):
        assert np.array_equal(shm[k].view(np.uint32), m.view(np.uint32))
    assert np.array_equal(cov, fr.cov)
    assert np.array_equal(tid, fr.tri_id)
    assert np.array_equal(db.view(np.uint32), fr.db.view(np.uint32))
    assert np.array_equal(r, fr.ro) and np.array_equal(g, fr.go) and np.array_equal(b, fr.bo)


@pytest.mark.parametrize("name", sorted(SCENES))
def test_kat_cuda_equals_oracle(name):
    sc = SCENES[name]
    mask = kat.masks(name, len(sc.groups))
    fr, smaps = oracle_frame(sc, VIEW, mask)
    got, _ = cuda_frame(sc, VIEW, mask)
    assert_same(fr, smaps, got)


def test_shadow_border_taps_cuda_equals_oracle():
    """Shadow lookups on and past a cascade's outer texels (kat's border
    scene): maps, coverage, ids and depth bit-exact, colour at the parity
    bar, and the shadow count read back from every covered pixel equal to
    the oracle's, on the tiled and the small path."""
    from test_gpu_parity import check_frame
    sc = kat.shadow_border_scene(VIEW.w, VIEW.h)
    smaps = []
    for k, s in enumerate(sc.shadows):
        m = O.new_shadow_map(s.dim)
        O.shadow_map(sc, k, m)
        smaps.append(m)
    fr = O.Frame(VIEW.w, VIEW.h)
    O.clear_depth(fr.db)
    O.draw_all(sc, VIEW, fr, smaps)
    got, _ = cuda_frame(sc, VIEW)
    check_frame(fr, smaps, got)
    cov = fr.cov.astype(bool)
    s_cuda, s_orc = kat.decode_shadow_count(got[0]), kat.decode_shadow_count(fr.ro)
    assert np.array_equal(s_cuda[cov], s_orc[cov])
    assert (s_orc[cov] == 5).any() and (s_orc[cov] == 0).any()


def test_trilinear_level_selection_cuda_equals_oracle():
    """kat's mip scene (mid-range level and upper clamp on the tiled path;
    lower clamp through a negative mipBias, dt > 1 and truncated vertices
    on the small path): coverage, ids and depth bit-exact, colour at the
    parity bar, and each pixel's level read back equal to the oracle's."""
    from test_gpu_parity import check_frame
    sc, view, cases = kat.mip_scene()
    fr = O.Frame(view.w, view.h)
    O.clear_depth(fr.db)
    O.draw_all(sc, view, fr, [])
    got, R = cuda_frame(sc, view)
    check_frame(fr, [], got)
    for k in range(len(cases)):
        px = fr.tri_id == k
        lv_cuda = got[0][px].astype(np.float64) / kat.MIP_LEVEL_VALUE - 1.0
        lv_orc = fr.ro[px].astype(np.float64) / kat.MIP_LEVEL_VALUE - 1.0
        assert np.abs(lv_cuda - lv_orc).max() <= 2e-3, k
    assert [float(b) for b in R.draw._mip_bias] == [float(np.float32(b)) for _, _, b in cases]


def test_unit_queue_overflow_falls_back_then_grows(monkeypatch):
    monkeypatch.setenv("AXR_UNIT_QUEUE", "16")
    sc = S.scene_small(seed=1, flags=S.MIP | S.SHADOW)
    view = S.default_view(320, 240, pos=(3, 2, -8))
    fr, smaps = O.render(sc, view)
    got, R = cuda_frame(sc, view)
    st = R.draw.lastStats()
    assert st["n_units"] > 16                        # the first frame overflowed ...
    assert_same(fr, smaps, got)                      # ... and the fallback drew it exactly
    R.frame(view)                                    # the queue has grown: the unit path again
    r, g, b, db = R.draw.getFrame()
    assert np.array_equal(db.view(np.uint32), fr.db.view(np.uint32))


def test_repeated_frames_are_identical():
    sc = S.scene_small(seed=2, flags=S.MIP | S.SHADOW)
    view = S.default_view(256, 192, pos=(1, 3, -12))
    got, R = cuda_frame(sc, view)
    for _ in range(3):
        R.frame(view)
    r, g, b, db = R.draw.getFrame()
    assert np.array_equal(db.view(np.uint32), got[3].view(np.uint32))
    assert np.array_equal(r, got[0])


def test_api_errors_raise():
    from axi_visualizer_b200._lib import AxrError
    from axi_visualizer_b200.ops import CLDraw, SceneRenderer
    with pytest.raises(AxrError):
        CLDraw(1, 64, 100, 64, 1)                    # width not a multiple of 16
    sc = S.scene_small(seed=1, flags=S.MIP | S.SHADOW)
    R = SceneRenderer(sc, 64, 48)
    with pytest.raises(AxrError):
        R.draw.drawAll(R.shaders[:-1])               # group count mismatch
    with pytest.raises(AxrError):
        R.draw.drawAll(R.shaders, shadowIds=[])      # shadow materials with no shadow map
    bad = list(R.shaders)
    bad[-1] = {"alpha": 5}
    with pytest.raises(AxrError):
        R.draw.drawAll(bad)                          # alpha mask index out of range
    with pytest.raises(AxrError):
        R.draw.addTextureGroup(np.zeros((4, 3)), np.zeros((4, 2)), np.zeros((4, 3)),
                               np.zeros(16), np.zeros(16), np.zeros(16))   # not 3 vertices per triangle
    # ranges whose int sum overflows are refused, not wrapped
    assert R.draw._L.axr_copy_to(R.draw._h, 0, None, None, 2**30, 2**31 - 1) != 0
    from axi_visualizer_b200.batch import Batch, shaded
    with pytest.raises(AxrError):
        Batch(R.draw, [shaded(S.default_view(64, 48), [], groups=(2**31 - 2, 5))])
    R.draw.drawAll(R.shaders)                        # the handle still works
    R.draw.sync()


def test_row_chunking_does_not_change_the_frame():
    """Small triangles and shadow casters are cut into row chunks (sorted by
    length at setup, alpha-tested casters at half length) whose lanes replay
    the row accumulation from the set-up slopes of both halves; every chunk
    size gives the same bits -- frame, triangle ids and both cascades -- on a
    scene with tall small triangles and alpha-tested quads, and the default
    equals the oracle."""
    from axi_visualizer_b200.ops import SceneRenderer
    sc = S.scene_small(seed=5, flags=S.MIP | S.SHADOW, nquads=120)
    view = S.default_view(480, 272, pos=(0, 4, -14))
    R = SceneRenderer(sc, view.w, view.h)
    frames = []
    for mc in (12, 1, 2, 4, 16, 32, 256):
        R.draw._L.axr_set_tuning(R.draw._h, mc)
        R.shadow_pass()
        R.set_view(view)
        R.draw.clearZBuffer()
        R.draw.drawAll(R.shaders, shadowIds=[0, 1])
        frames.append([x.copy() for x in R.draw.getFrame()] + [R.draw.getIDs()[0]] +
                      [R.draw.getSHM(k) for k in range(len(sc.shadows))])
    fr, smaps = O.render(sc, view)
    for k, m in enumerate(smaps):
        assert np.array_equal(frames[0][5 + k].view(np.uint32), m.view(np.uint32)), f"cascade {k}"
    assert np.array_equal(frames[0][3].view(np.uint32), fr.db.view(np.uint32))
    assert np.array_equal(frames[0][4], fr.tri_id)
    st = R.draw.lastStats()
    assert st["n_small"] > 0
    for f in frames[1:]:
        for a, b in zip(f, frames[0]):
            assert np.array_equal(a.view(np.uint8), b.view(np.uint8))


def test_async_frame_read_equals_get_frame():
    """readFrameAsync / waitFrame deliver the same frame as getFrame, also
    with two reads in flight and the next frames rendering meanwhile."""
    sc = S.scene_small(seed=2, flags=S.MIP | S.SHADOW)
    views = [S.default_view(256, 192, pos=p) for p in ((1, 3, -12), (4, 2, -9), (-3, 5, -10))]
    from axi_visualizer_b200.ops import SceneRenderer
    R = SceneRenderer(sc, 256, 192, pinned=True)
    want = []
    for v in views:
        R.draw.clearColor((1, 1, 1))           # uncovered pixels would keep the previous frame's colour
        R.frame(v)
        want.append([x.copy() for x in R.draw.getFrame()])
    tickets = []
    for rep in range(2):
        for k, v in enumerate(views):
            R.draw.clearColor((1, 1, 1))
            R.frame(v)
            tickets.append((k, R.draw.readFrameAsync()))
            if len(tickets) >= 2:              # at most two reads in flight
                kk, t = tickets.pop(0)
                got = R.draw.waitFrame(t)
                for a, b in zip(got, want[kk]):
                    assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
    for kk, t in tickets:
        got = R.draw.waitFrame(t)
        assert R.draw.frameDone(t)
        for a, b in zip(got, want[kk]):
            assert np.array_equal(a.view(np.uint8), b.view(np.uint8))


def test_rgb8_read_back_equals_gamma_of_the_planes():
    """readFrameRGB8Async packs Post/gamma.c's mapping of the colour planes
    as interleaved 8-bit RGB on the device: equal to the oracle's gamma of
    the same planes, for two exposures, and the planes stay unchanged."""
    from axi_visualizer_b200.ops import SceneRenderer
    sc = S.scene_small(seed=4, flags=S.MIP | S.SHADOW)
    view = S.default_view(320, 240, pos=(3, 2, -8))
    R = SceneRenderer(sc, 320, 240, pinned=True)
    R.frame(view)
    planes = [x.copy() for x in R.draw.getFrame()[:3]]
    for ex in (1.0, 0.37):
        t = R.draw.readFrameRGB8Async(ex)
        rgb = R.draw.waitFrame(t).copy()
        fr = O.Frame(320, 240)
        fr.ro, fr.go, fr.bo = (p.copy() for p in planes)
        O.gamma(fr, ex)
        want = np.stack((fr.ro, fr.go, fr.bo), axis=-1).astype(np.uint8)
        assert rgb.shape == (240, 320, 3) and np.array_equal(rgb, want)
    after = R.draw.getFrame()[:3]
    for a, b in zip(after, planes):
        assert np.array_equal(a, b)
