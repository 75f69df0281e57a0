"""The named workloads at their full sizes on the GPU.

- 1920x1080 / 1,044,288 triangles (terrain, icospheres, alpha-tested quads,
  trilinear 2048^2 textures, two 2048^2 cascades): CUDA frame against the
  oracle (OpenMP), same bars as the small parity cases -- coverage, triangle
  ids, depth and shadow maps bit-exact, colour within 1/255 after gamma.
- 3840x2160 / 9,988,608 triangles: the CUDA frame and both 4096^2 cascades
  against the oracle at the same bars, and the batched launch of the
  cascades, the main view and six cube faces against the plain path.
- The batched view set of the 24,192-triangle scene (six 512^2 cube faces,
  2048^2 + 1024^2 cascades, the 1920x1080 main view) in one persistent
  launch: every view bit-identical to the same view rendered alone.
"""
import os

import numpy as np
import pytest

import oracle as O
from axi_visualizer_b200 import scenes as S

from test_gpu_parity import check_frame

pytestmark = pytest.mark.gpu


def test_1080p_1m_triangle_frame_equals_oracle():
    from axi_visualizer_b200.ops import SceneRenderer
    sc = S.scene_c2()
    view = S.default_view(1920, 1080)
    fr, smaps = O.render(sc, view, nthreads=os.cpu_count() or 1)
    R = SceneRenderer(sc, 1920, 1080)
    R.frame(view)
    r, g, b, db = [x.copy() for x in R.draw.getFrame()]
    tid, cov = R.draw.getIDs()
    shm = [R.draw.getSHM(k) for k in range(len(sc.shadows))]
    exact, psnr = check_frame(fr, smaps, (r, g, b, db, tid, cov, shm))
    st = R.draw.lastStats()
    assert st["n_small"] > 300_000 and st["n_units"] > 100_000
    assert (tid >= 0).mean() > 0.5                  # most of the frame is covered
    print(f"1080p/1M: exact u16 fraction {exact:.6f}, PSNR {psnr:.1f} dB")


def test_batched_view_set_equals_single_views():
    from axi_visualizer_b200.batch import Batch, cube_faces, scene_batch_views
    from axi_visualizer_b200.ops import SceneRenderer
    sc = S.scene_c3()
    main = S.default_view(1920, 1080)
    eye = (0.0, 5.0, -25.0)
    R = SceneRenderer(sc, 1920, 1080)
    descs = scene_batch_views(sc, main, faces_at=eye, face_side=512)
    assert [d.w for d in descs] == [2048, 1024, 1920] + [512] * 6
    B = Batch(R.draw, descs)
    flags = [g.flags for g in sc.groups]
    aidx = [g.alpha_index for g in sc.groups]
    B.render(flags, aidx)
    B.render(flags, aidx)                            # graph replay
    R.shadow_pass()
    nd = len(sc.shadows)
    for k in range(nd):
        assert np.array_equal(B.frame(k).view(np.uint32), R.draw.getSHM(k).view(np.uint32))
    casc = list(range(nd))
    R.set_view(main)
    R.draw.clearZBuffer()
    R.draw.drawAll(R.shaders, shadowIds=casc)
    want = [x.copy() for x in R.draw.getFrame()]
    got = B.frame(nd)
    for a, w in zip(got, want):
        assert np.array_equal(a.view(np.uint8), w.view(np.uint8))
    assert np.array_equal(B.ids(nd)[0], R.draw.getIDs()[0])
    F = SceneRenderer(sc, 512, 512)
    F.shadow_pass()
    for j, fv in enumerate(cube_faces(eye, 512)):
        F.set_view(fv)
        F.draw.clearZBuffer()
        F.draw.clearColor((1, 1, 1))                 # a face's slot in the batch never held another face
        F.draw.drawAll(F.shaders, shadowIds=casc)
        want = [x.copy() for x in F.draw.getFrame()]
        got = B.frame(nd + 1 + j)
        for a, w in zip(got, want):
            assert np.array_equal(a.view(np.uint8), w.view(np.uint8)), f"cube face {j}"
    assert B.stats()["graph"]


def test_stress_scene_equals_oracle_and_batched_launch():
    """3840x2160 / 9,988,608 triangles, 16 trilinear 4096^2 textures, 29%
    alpha-tested, 4096^2 cascades: the plain shadowMap + drawAll frame
    against the oracle (OpenMP, all host cores) at the parity bars --
    coverage, triangle ids, depth and both cascades bit-exact, colour within
    1/255 after gamma -- and the batched launch of both cascades, the main
    view and six 1024^2 cube faces bit for bit as the plain path."""
    from axi_visualizer_b200.batch import Batch, scene_batch_views
    from axi_visualizer_b200.ops import SceneRenderer
    sc = S.scene_c5()
    assert sc.ntris == 9_988_608 and len(sc.groups) == 16
    main = S.default_view(3840, 2160, pos=(0.0, 8.0, -40.0))
    R = SceneRenderer(sc, 3840, 2160)
    descs = scene_batch_views(sc, main, faces_at=(0.0, 8.0, -30.0), face_side=1024)
    B = Batch(R.draw, descs)
    B.render([g.flags for g in sc.groups], [g.alpha_index for g in sc.groups])
    R.frame(main)
    nd = len(sc.shadows)
    for k in range(nd):
        assert np.array_equal(B.frame(k).view(np.uint32), R.draw.getSHM(k).view(np.uint32)), f"cascade {k}"
    want = [x.copy() for x in R.draw.getFrame()]
    tid, cov = R.draw.getIDs()
    got = B.frame(nd)
    for a, w in zip(got, want):
        assert np.array_equal(a.view(np.uint8), w.view(np.uint8))
    assert np.array_equal(B.ids(nd)[0], tid)
    st = R.draw.lastStats()
    assert st["n_small"] > 1_000_000 and cov.mean() > 0.5
    fr, smaps = O.render(sc, main, nthreads=os.cpu_count() or 1)
    shm = [R.draw.getSHM(k) for k in range(nd)]
    exact, psnr = check_frame(fr, smaps, (*want, tid, cov, shm))
    print(f"4K/10M: exact u16 fraction {exact:.6f}, PSNR {psnr:.1f} dB")
