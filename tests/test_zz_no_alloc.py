"""axr_shadow_map_noalloc against axr_shadow_map.

The no-allocation entry point is for callers that cannot call
cudaMalloc/cudaFree while rendering (their own allocator owns all device
memory, or their frame loop must not take the implicit device
synchronisation those calls can cause).  It keeps its scratch in a fixed
array inside libaxr.so, so this test checks that two calls in a row (the
second one starting from the scratch contents the first left behind) give
the same depth maps, bit for bit, as the handle-based entry point on the
same casters.  The test allocates its own device buffers with torch; the
entry point under test allocates nothing.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from axi_visualizer_b200 import scenes as S

pytestmark = pytest.mark.gpu


def _handle_map(sc, k, group):
    """Depth map of `group`'s triangles through the handle-based entry point."""
    from axi_visualizer_b200.ops import SceneRenderer
    R = SceneRenderer(sc, 64, 64)
    cast = [i == group for i in range(len(sc.groups))]
    R.draw.clearShadowMap(k)
    R.draw.shadowMap(k, cast, R.shaders, sc.bias)
    return R.draw.getSHM(k)


def test_noalloc_shadow_two_calls_match_handle_path():
    import torch
    from axi_visualizer_b200._lib import check, lib

    L = lib()
    sc = S.scene_small(seed=5, flags=0, with_alpha=True)
    dev = torch.device("cuda:0")
    torch.cuda.set_device(0)
    # call 1: opaque terrain into cascade 0; call 2: alpha-tested quads into cascade 1
    for k, group in ((0, 0), (1, 2)):
        want = _handle_map(sc, k, group)
        g = sc.groups[group]
        cam = sc.shadows[k]
        xyz = torch.from_numpy(np.ascontiguousarray(g.xyz)).to(dev)
        uv = torch.from_numpy(np.ascontiguousarray(g.uv)).to(dev)
        mask = None
        side = 0
        if g.flags & S.ALPHA:
            m, side = sc.alphas[g.alpha_index]
            mask = torch.from_numpy(np.ascontiguousarray(m, np.uint8)).to(dev)
        out = torch.full((cam.dim, cam.dim), 65535.0, dtype=torch.float32, device=dev)
        pos = np.ascontiguousarray(cam.pos, np.float32)
        vm = np.ascontiguousarray(np.asarray(cam.vv, np.float32).reshape(9))
        stream = torch.cuda.current_stream(dev)
        check(L.axr_shadow_map_noalloc(xyz.data_ptr(), uv.data_ptr(), mask.data_ptr() if mask is not None else None,
                                       side, g.ntris, pos.ctypes.data, vm.ctypes.data, C.c_float(cam.scale),
                                       C.c_float(sc.bias), out.data_ptr(), cam.dim, C.c_void_p(stream.cuda_stream)),
              "axr_shadow_map_noalloc")
        torch.cuda.synchronize(dev)
        got = out.cpu().numpy()
        assert (got < 65535).sum() > 0, "no texel written"
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), \
            f"call {k + 1}: {(got != want).sum()} texels differ from axr_shadow_map"


def test_noalloc_rejects_oversize_input():
    from axi_visualizer_b200._lib import lib
    L = lib()
    pos = np.zeros(3, np.float32)
    vm = np.eye(3, dtype=np.float32).reshape(9)
    rc = L.axr_shadow_map_noalloc(C.c_void_p(16), None, None, 0, (1 << 20) + 1, pos.ctypes.data, vm.ctypes.data,
                                  C.c_float(1.0), C.c_float(0.0), C.c_void_p(16), 64, None)
    assert rc != 0
    assert b"at most 1048576 triangles" in L.axr_last_error()
