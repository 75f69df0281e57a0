"""Serving on the GPU: every request's frame is the same rendered in the mix
(continuous batching over resident scenes, several slabs in flight) as
rendered alone, through the plain per-view path, and in a handle holding its
scene alone.  Tolerance: bit-exact colour planes and depth (the stated bar is
1/255 after gamma; these paths share all arithmetic, so nothing differs)."""
import numpy as np
import pytest

from axi_visualizer_b200 import scenes as S
from axi_visualizer_b200 import serve as SV

pytestmark = pytest.mark.gpu

RES = ((160, 96), (320, 176), (480, 272))
LAYOUT = {RES[0]: 3, RES[1]: 2, RES[2]: 1}


@pytest.fixture(scope="module")
def world():
    scenes = [S.scene_served(s, tmin=2_000, tmax=20_000, tex=64, alpha_tex=64, cascades=(256, 128))
              for s in (10, 11, 12)]
    return scenes, SV.ResidentScenes(scenes)


def trace(burst=True, n=16):
    return SV.poisson_trace(n, 2000.0, 3, seed=5, resolutions=RES, probs=(0.4, 0.35, 0.25), burst=burst)


def frames(tr):
    return {r.rid: r.frame for r in tr}


def same(a, b, rid):
    for k, name in enumerate(("r", "g", "b", "depth")):
        assert a[k].shape == b[k].shape, (rid, name)
        assert np.array_equal(a[k].view(np.uint8), b[k].view(np.uint8)), f"request {rid}: {name} differs"


def test_mix_equals_alone(world):
    scenes, res = world
    mix = trace()
    srv = SV.Server(SV.GpuBackend(res), layout=LAYOUT, max_slabs=3, depth=2, keep_frames=True)
    st = srv.run(mix, timeout=120)
    assert st["done"] == len(mix), st
    assert max(srv.launch_sizes) > 1 and st["max_inflight"] == 2     # batched, and overlapped
    assert len({r.scene for r in mix if r.launch_id == mix[0].launch_id}) >= 1
    # several scenes within one launch
    by_launch = {}
    for r in mix:
        by_launch.setdefault(r.launch_id, set()).add(r.scene)
    assert max(len(v) for v in by_launch.values()) > 1

    alone_be = SV.GpuBackend(res)
    for r in trace():
        one = SV.Server(alone_be, layout=LAYOUT, max_slabs=1, depth=1, keep_frames=True)
        assert one.run([r], timeout=60)["done"] == 1
        one.close()
        same(frames(mix)[r.rid], r.frame, r.rid)
    srv.close()


def test_mix_equals_plain_path_and_own_handle(world):
    scenes, res = world
    mix = trace(burst=False)
    srv = SV.Server(SV.GpuBackend(res), layout=LAYOUT, max_slabs=2, depth=2, keep_frames=True)
    assert srv.run(mix, timeout=120)["done"] == len(mix)
    srv.close()
    plain = trace(burst=False)
    st = SV.PlainServer(scenes, RES).run(plain, keep_frames=True)
    assert st["done"] == len(plain)
    for a, b in zip(mix, plain):
        same(a.frame, b.frame, a.rid)
    from axi_visualizer_b200.ops import SKY_COLOR, SceneRenderer
    assert SKY_COLOR == SV.SKY
    for r in mix[:4]:
        own = SceneRenderer(scenes[r.scene], r.w, r.h)
        own.shadow_pass()
        own.set_view(r.view())
        own.draw.clearZBuffer()
        own.draw.clearColor(SKY_COLOR)
        own.draw.drawAll(own.shaders, shadowIds=[0, 1])
        same(r.frame, own.draw.getFrame(), r.rid)
        # pixels no triangle covers hold the sky colour
        cov = own.draw.getIDs()[1]
        if (cov == 0).any():
            assert (r.frame[0][cov == 0] == SKY_COLOR[0]).all()


def test_slab_bytes_match_the_library(world):
    _, res = world
    be = SV.GpuBackend(res)
    slots = [wh for wh, n in LAYOUT.items() for _ in range(n)]
    h = be.create(slots)
    actual = h["batch"].bytes()
    est = be.slab_bytes(slots)
    assert abs(est - actual) < (1 << 20) and est >= actual
    be.destroy(h)
