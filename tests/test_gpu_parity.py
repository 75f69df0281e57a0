"""CUDA path (libaxr.so through the C ABI) against the CPU oracle.

Bars: coverage and triangle ids bit-exact; depth bit-exact (<= 1 ulp is the
stated tolerance, the implementation reaches 0); shadow maps bit-exact;
colour after Post/gamma.c (exposure 1, 8-bit range) within 1/255 max-abs per
channel, with PSNR and the exact-match fraction of the raw u16 planes.
"""
import numpy as np
import pytest

import oracle as O
from axi_visualizer_b200 import scenes as S

pytestmark = pytest.mark.gpu

COLOR_TOL = 1  # max abs difference on the 0..255 gamma-mapped channels (= 1/255)


def _ulps(a, b):
    ai = a.view(np.int32).astype(np.int64)
    bi = b.view(np.int32).astype(np.int64)
    ai = np.where(ai < 0, -(ai & 0x7fffffff), ai)
    bi = np.where(bi < 0, -(bi & 0x7fffffff), bi)
    return np.abs(ai - bi)


def _psnr(a, b):
    mse = np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2)
    return float("inf") if mse == 0 else 10 * np.log10(255.0 ** 2 / mse)


def render_both(sc, view):
    from axi_visualizer_b200.ops import SceneRenderer
    fr, smaps = O.render(sc, view)
    R = SceneRenderer(sc, view.w, view.h)
    R.frame(view)
    r, g, b, db = [x.copy() for x in R.draw.getFrame()]
    tid, cov = R.draw.getIDs()
    shm = [R.draw.getSHM(k) for k in range(len(sc.shadows))]
    return fr, smaps, (r, g, b, db, tid, cov, shm), R


def check_frame(fr, smaps, got, R=None):
    r, g, b, db, tid, cov, shm = got
    for k, m in enumerate(smaps):
        assert np.array_equal(shm[k].view(np.uint32), m.view(np.uint32)), f"shadow map {k}: {(shm[k] != m).sum()} px differ"
    assert np.array_equal(cov, fr.cov), f"coverage: {(cov != fr.cov).sum()} px differ"
    assert np.array_equal(tid, fr.tri_id), f"triangle id: {(tid != fr.tri_id).sum()} px differ"
    assert _ulps(db, fr.db).max() <= 1
    assert np.array_equal(db.view(np.uint32), fr.db.view(np.uint32))
    exact = np.mean((r == fr.ro) & (g == fr.go) & (b == fr.bo))
    # 8-bit comparison through Post/gamma.c on both sides
    og = O.Frame(fr.w, fr.h)
    og.ro, og.go, og.bo = fr.ro.copy(), fr.go.copy(), fr.bo.copy()
    O.gamma(og)
    cg = O.Frame(fr.w, fr.h)
    cg.ro, cg.go, cg.bo = r.copy(), g.copy(), b.copy()
    O.gamma(cg)
    diff = max(int(np.abs(og.ro.astype(int) - cg.ro).max()), int(np.abs(og.go.astype(int) - cg.go).max()),
               int(np.abs(og.bo.astype(int) - cg.bo).max()))
    assert diff <= COLOR_TOL, f"colour max abs {diff}/255"
    return exact, _psnr(np.stack((og.ro, og.go, og.bo)), np.stack((cg.ro, cg.go, cg.bo)))


VIEWS = [(0, 8, -30), (3, 2, -8), (0, 30, -1), (-20, 3, 5)]


@pytest.mark.parametrize("flags", [0, S.MIP, S.SHADOW, S.MIP | S.SHADOW])
@pytest.mark.parametrize("pos", VIEWS)
def test_small_scene_parity(flags, pos):
    sc = S.scene_small(seed=3, flags=flags)
    view = S.default_view(320, 240, pos=pos)
    fr, smaps, got, _ = render_both(sc, view)
    exact, psnr = check_frame(fr, smaps, got)
    assert exact > 0.999


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_seeds_and_resolutions(seed):
    sc = S.scene_small(seed=seed, flags=S.MIP | S.SHADOW)
    for (w, h) in [(160, 120), (256, 200), (640, 360)]:
        view = S.default_view(w, h, pos=(2.0 * seed, 5, -20))
        fr, smaps, got, _ = render_both(sc, view)
        check_frame(fr, smaps, got)


def test_c1_scene_parity():
    sc = S.scene_c1()
    view = S.default_view(640, 480)
    fr, smaps, got, R = render_both(sc, view)
    exact, psnr = check_frame(fr, smaps, got)
    st = R.draw.lastStats()
    assert st["n_small"] > 0


@pytest.mark.parametrize("pos", [(0, 8, -20), (4, 3, -6)])
def test_alpha_tested_trilinear_materials(pos):
    """The composed material in full (alpha test, trilinear mip, double
    cascade), with and without culling, as the 3840x2160 stress scene uses
    it, on a miniature of that scene (64x64 terrain in 4 bands, 300
    icospheres, 64^2 textures and mask, 512^2 + 256^2 cascades): against
    the oracle at the parity bars."""
    sc = S.scene_c5(seed=7, terrain_n=64, spheres=300, tex=64, terrain_groups=4, sphere_groups=2,
                    alpha_terrain=(1, 2), alpha_spheres=(0,), cascades=(512, 256), extent=16.0)
    view = S.default_view(320, 240, pos=pos)
    fr, smaps, got, R = render_both(sc, view)
    exact, psnr = check_frame(fr, smaps, got)
    base = np.cumsum([0] + [g.ntris for g in sc.groups])
    composed = np.zeros(fr.cov.shape, bool)
    for k, g in enumerate(sc.groups):
        if g.flags & S.ALPHA and g.flags & S.MIP:
            composed |= (fr.tri_id >= base[k]) & (fr.tri_id < base[k + 1])
    assert composed.sum() > 1000
    assert exact > 0.999
