"""The oracle pinned to the reference: golden fixtures made by the
reference's own kernels (tests/golden/make_golden.py), and -- where
oracle/_ref is built -- the reference kernels run live on the same inputs.
Bit-exact on depth, colour and shadow maps."""
import hashlib
import os
import sys
import types

import numpy as np
import pytest

import oracle as O
from axi_visualizer_b200 import scenes as S

GOLD = os.path.join(os.path.dirname(__file__), "golden")
CASES = [(3, 160, 120, (0, 8, -30)), (1, 160, 128, (3, 2, -8)), (2, 128, 96, (-20, 3, 5))]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(GOLD, "ref_frames.npz"))


@pytest.mark.parametrize("i", range(len(CASES)))
def test_oracle_equals_reference_golden_frames(gold, i):
    seed, w, h, pos = CASES[i]
    sc = S.scene_small(seed=seed, flags=0, with_alpha=True)
    fr, smaps = O.render(sc, S.default_view(w, h, pos=pos))
    for k, m in enumerate(smaps):
        assert np.array_equal(m.view(np.uint32), gold[f"c{i}_shm{k}"].view(np.uint32))
    assert np.array_equal(fr.db.view(np.uint32), gold[f"c{i}_db"].view(np.uint32))
    for n, a in (("r", fr.ro), ("g", fr.go), ("b", fr.bo)):
        assert np.array_equal(a, gold[f"c{i}_{n}"])
        assert sha(a) == str(gold[f"c{i}_{n}_sha256"])


def test_oracle_equals_reference_golden_1080p_scene(gold):
    """1,044,288 triangles at 1920x1080 with two 2048^2 cascades, through the
    reference kernels' materials (bilinear base level, alpha test)."""
    sc = S.reference_kernel_variant(S.scene_c2())
    fr, smaps = O.render(sc, S.default_view(1920, 1080), nthreads=os.cpu_count() or 1)
    for k, m in enumerate(smaps):
        assert sha(m) == str(gold[f"hd_shm{k}_sha256"])
    for n, a in (("r", fr.ro), ("g", fr.go), ("b", fr.bo), ("db", fr.db)):
        assert sha(a) == str(gold[f"hd_{n}_sha256"]), n


needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("seed", [0, 4])
@pytest.mark.parametrize("pos", [(0, 8, -30), (3, 2, -8), (0, 30, -1), (-20, 3, 5), (6, 1.5, -4)])
def test_oracle_equals_reference_kernels_live(seed, pos):
    sc = S.scene_small(seed=seed, flags=0, with_alpha=True)
    view = S.default_view(192, 144, pos=pos)
    fr, smaps = O.render(sc, view)
    rd = O.RefDraw(sc, view)
    for k in range(len(sc.shadows)):
        rc, m = rd.shadow_map(k)
        assert rc == 0 and np.array_equal(m.view(np.uint32), smaps[k].view(np.uint32))
    rd.clear_zbuffer()
    assert rd.draw_all() == 0
    r, g, b, db = rd.get_frame()
    assert np.array_equal(db.view(np.uint32), fr.db.view(np.uint32))
    assert np.array_equal(r, fr.ro) and np.array_equal(g, fr.go) and np.array_equal(b, fr.bo)


@needs_ref
def test_gamma_and_clear_match_reference():
    sc = S.scene_small(seed=1, flags=0)
    view = S.default_view(160, 120, pos=(3, 2, -8))
    rd = O.RefDraw(sc, view)
    rd.clear_zbuffer()
    rd.draw_all()
    rd.gamma(1.0)
    r, g, b, _ = rd.get_frame()
    fr, _ = O.render(sc, view)
    O.gamma(fr, 1.0)
    assert np.array_equal(r, fr.ro) and np.array_equal(g, fr.go) and np.array_equal(b, fr.bo)
    # clearzb over 4x4 work-items leaves the rows/columns past w/4*4, h/4*4
    d = np.zeros((18, 22), np.float32)
    O.clear_depth(d, 4)
    assert (d[:16, :20] == 65535).all() and (d[16:] == 0).all() and (d[:, 20:] == 0).all()


def test_scene_terrain_matches_reference_vertterrain():
    z = np.load(os.path.join(GOLD, "ref_terrain.npz"))
    h = z["heights"]
    xyz, vn, uv = S.terrain_from_heights(h, 1.0, (-2.0, 0.0, -2.0), uvspread=2.0)
    assert np.allclose(xyz, z["xyz"], atol=0, rtol=0)
    assert np.allclose(uv[:, 0], z["u"], atol=1e-15) and np.allclose(uv[:, 1], z["v"], atol=1e-15)


def test_create_mips_matches_reference():
    z = np.load(os.path.join(GOLD, "ref_terrain.npz"))
    assert np.array_equal(S.create_mips(z["tex"]), z["mips"])


# ---------------------------------------------------------------- 4-way blend material

def _multi_cases():
    sys.path.insert(0, GOLD)
    import make_golden as MG
    return MG.MULTI_CASES


@pytest.mark.parametrize("i", range(3))
def test_multi_material_equals_reference_golden(i):
    """av_draw_multi.c through the reference's own drawmulti.c kernels
    (tests/golden/ref_multi.npz) against the oracle: bit-exact."""
    gold = np.load(os.path.join(GOLD, "ref_multi.npz"))
    seed, w, h, pos, target = _multi_cases()[i]
    sc = S.reference_kernel_variant(S.scene_multi(seed=seed))
    fr, _ = O.render(sc, S.default_view(w, h, pos=pos, target=target))
    for n, a in (("r", fr.ro), ("g", fr.go), ("b", fr.bo), ("db", fr.db)):
        assert sha(a) == str(gold[f"m{i}_{n}_sha256"]), n


@needs_ref
@pytest.mark.parametrize("seed", [9, 11])
@pytest.mark.parametrize("pos", [(0, 30, -40), (-10, 8, -12), (12, 4, 6)])
def test_multi_material_equals_reference_kernels_live(seed, pos):
    sc = S.reference_kernel_variant(S.scene_multi(seed=seed))
    view = S.default_view(160, 128, pos=pos, target=(0, 12, 0))
    fr, _ = O.render(sc, view)
    rd = O.RefDraw(sc, view)
    rd.clear_zbuffer()
    assert rd.draw_all() == 0
    r, g, b, db = rd.get_frame()
    assert np.array_equal(db.view(np.uint32), fr.db.view(np.uint32))
    assert np.array_equal(r, fr.ro) and np.array_equal(g, fr.go) and np.array_equal(b, fr.bo)
    terrain = (fr.tri_id >= 0) & (fr.tri_id < sc.groups[0].ntris)
    assert terrain.sum() > 1000 or pos == (12, 4, 6)


def _mip_pin_scenes():
    """Scenes of trilinear materials only (no alpha, no shadow lookup):
    kat's level-selection cases, and seeded terrain + spheres with mipBias
    0, 0.7 and -0.4."""
    import kat
    out = [kat.mip_scene()[:2]]
    for seed, bias in ((3, 0.0), (8, 0.7), (12, -0.4)):
        sc = S.scene_small(seed=seed, flags=S.MIP, with_alpha=False)
        for g in sc.groups:
            g.mip_bias = bias
        out.append((sc, S.default_view(160, 120, pos=(2, 6, -14))))
    return out


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (needs the reference checkout)")
@pytest.mark.parametrize("i", range(4))
def test_trilinear_core_equals_reference_mip_material(i):
    """The oracle's trilinear colour against the reference's own code: its
    normal-mapped mip material (Shaders_src/av_draw_normmap_mip.c, expanded
    by the reference's AVSL generator, tiled and small kernels) drawn with a
    zero light intensity, where its colour is exactly the trilinear texel
    (level selection :26-59, both bilinear taps and the blend :73-123) times
    the interpolated vertex light -- the composed material's colour with the
    same zero intensity.  Depth and all three u16 planes bit for bit."""
    sc, view = _mip_pin_scenes()[i]
    sc.lint = np.zeros(3, np.float32)
    fr = O.Frame(view.w, view.h)
    O.clear_depth(fr.db)
    O.draw_all(sc, view, fr)
    rd = O.RefDraw(sc, view)
    rd.set_mip_kernels(True)
    rd.clear_zbuffer()
    assert rd.draw_all() == 0
    r, g, b, db = rd.get_frame()
    assert (db < 65535).sum() > 500, "the scene covers the frame"
    assert np.array_equal(db.view(np.uint32), fr.db.view(np.uint32)), "depth differs"
    for n, a, o in (("r", r, fr.ro), ("g", g, fr.go), ("b", b, fr.bo)):
        d = int((a != o).sum())
        assert d == 0, f"{n}: {d} px differ (max {int(np.abs(a.astype(int) - o).max())})"


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (needs the reference checkout)")
@pytest.mark.parametrize("seed,pos", [(6, (2, 6, -14)), (13, (-4, 9, -10))])
def test_normal_mapped_materials_equal_reference_kernels(seed, pos):
    """The oracle's normal-mapped materials against the reference's own
    kernels (Shaders_src/av_draw_normmap.c, _alpha.c and _mip.c expanded by
    its AVSL generator, tiled and small): tangent frames, normal-map taps,
    the specular terms, the metal switch, the alpha test and the trilinear
    chain, with the light on and the first cascade sampled.  The reference
    defines sampleShadow nowhere; both sides use this library's definition.
    Depth and all three u16 planes bit for bit."""
    sc = S.scene_normal(seed=seed)
    view = S.default_view(160, 120, pos=pos)
    fr, smaps = O.render(sc, view)
    rd = O.RefDraw(sc, view)
    for k in range(len(sc.shadows)):
        rc, m = rd.shadow_map(k)
        assert rc == 0 and np.array_equal(m.view(np.uint32), smaps[k].view(np.uint32))
    rd.clear_zbuffer()
    assert rd.draw_all() == 0
    r, g, b, db = rd.get_frame()
    covered = fr.cov.astype(bool)
    assert covered.sum() > 2000, "the scene covers the frame"
    for gi in range(len(sc.groups)):
        base = sum(x.ntris for x in sc.groups[:gi])
        assert ((fr.tri_id >= base) & (fr.tri_id < base + sc.groups[gi].ntris)).any(), f"group {gi} visible"
    assert np.array_equal(db.view(np.uint32), fr.db.view(np.uint32)), "depth differs"
    for n, a, o in (("r", r, fr.ro), ("g", g, fr.go), ("b", b, fr.bo)):
        d = int((a != o).sum())
        assert d == 0, f"{n}: {d} px differ (max {int(np.abs(a.astype(int) - o).max())})"
