"""Edge cases on the CPU: the oracle against the reference's own kernels
(oracle/_ref) on authored known-answer scenes (tests/kat.py)."""
import numpy as np
import pytest

import kat
import oracle as O

SCENES, VIEW = kat.case_scenes()
needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")


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


@needs_ref
@pytest.mark.parametrize("name", sorted(SCENES))
def test_kat_oracle_equals_reference(name):
    sc = SCENES[name]
    mask = kat.masks(name, len(sc.groups))
    fr, smaps = oracle_frame(sc, VIEW, mask)
    rd = O.RefDraw(sc, VIEW)
    for k in range(len(sc.shadows)):
        rc, m = rd.shadow_map(k)
        assert rc == 0
        assert np.array_equal(m.view(np.uint32), smaps[k].view(np.uint32))
    rd.clear_zbuffer()
    rc = rd.draw_all(mask=mask)
    if name == "bin_overflow":
        # the reference's 128-entry tile bins overflow (undefined there);
        # the oracle keeps every entry
        assert rc == -2
        assert fr.cov.sum() > 0
        return
    assert rc == 0
    r, g, b, db = rd.get_frame()
    assert np.array_equal(db.view(np.uint32), fr.db.view(np.uint32))
    assert np.array_equal(r, fr.ro) and np.array_equal(g, fr.go) and np.array_equal(b, fr.bo)


def test_kat_expectations():
    """Facts about the cases that do not depend on the reference."""
    fr, _ = oracle_frame(SCENES["near_plane"], VIEW)
    ids = set(np.unique(fr.tri_id[fr.tri_id >= 0]).tolist())
    assert ids == {2}, "triangles crossing the near plane are dropped whole"
    fr, _ = oracle_frame(SCENES["slivers"], VIEW)
    assert 0 not in set(np.unique(fr.tri_id).tolist()), "zero-size integer bbox is rejected"
    # exact depth ties: the later fragment in (pass, material, triangle) order wins
    sc = SCENES["depth_ties"]
    fr, _ = oracle_frame(sc, VIEW)
    ntri0 = sc.groups[0].ntris
    # the large copy (group 1, triangle 1 -> id ntri0+1) is drawn in the large
    # pass, after every small triangle, and covers the small ones at equal depth
    assert (fr.tri_id == ntri0 + 1).sum() > 0
    fr, _ = oracle_frame(SCENES["masked_empty"], VIEW, kat.masks("masked_empty", 3))
    ids = np.unique(fr.tri_id[fr.tri_id >= 0])
    assert ids.size and ids.min() >= SCENES["masked_empty"].groups[0].ntris + SCENES["masked_empty"].groups[1].ntris
    # rows at and below 16 * floor(h/16) are reached by small triangles only:
    # the large triangle of tile_borders covers the whole view but gives way
    # there to the small ones or to nothing
    sc = SCENES["tile_borders"]
    fr, _ = oracle_frame(sc, VIEW)
    top = 16 * (VIEW.h // 16)
    assert top < VIEW.h
    assert (fr.tri_id[:top] == 3).sum() > 0
    assert not (fr.tri_id[top:] == 3).any()
    assert (fr.tri_id[top:] >= 0).any()


def border_frame():
    sc = kat.shadow_border_scene(VIEW.w, VIEW.h)
    maps = []
    for k, s in enumerate(sc.shadows):
        m = O.new_shadow_map(s.dim)
        O.shadow_map(sc, k, m)
        maps.append(m)
    fr = O.Frame(VIEW.w, VIEW.h)
    O.clear_depth(fr.db)
    O.draw_all(sc, VIEW, fr, maps)
    return sc, fr, maps


def test_shadow_border_taps():
    """Shadow lookups at a cascade's border (av_alpha_max.c:53-84) on the
    oracle.  The count read back from each pixel clear of tap rounding is the
    one the rule gives from the maps.  Where cascade 0's centre tap falls on
    its two outer rows or columns, over texels the caster covers, with
    cascade 1 out of reach, the count is 0, on the tiled and the small path."""
    sc, fr, maps = border_frame()
    cov = fr.cov.astype(bool)
    s = kat.decode_shadow_count(fr.ro)
    want, clear, exposed = kat.border_counts(sc, maps, fr.tri_id, VIEW.w, VIEW.h)
    sel = cov & clear
    assert sel.sum() > 0.75 * cov.sum()
    assert np.array_equal(s[sel], want[sel])
    assert set(np.unique(s[cov]).tolist()) >= {0, 2, 3, 5}
    n0 = sc.groups[0].ntris
    small = (fr.tri_id >= n0) & (fr.tri_id < n0 + sc.groups[1].ntris)
    for path in (small, ~small):
        ex = sel & exposed & path
        assert ex.sum() >= 20
        assert not s[ex].any()
        assert (s[sel & path] == 5).any()
    # the caster is behind the camera: the view drops it, the maps hold it
    assert not (fr.tri_id >= n0 + sc.groups[1].ntris).any()
    assert all((m < 16.0).sum() > 0 for m in maps)


@needs_ref
def test_shadow_border_maps_and_depth_equal_reference():
    """The border scene's cascades through drawmin.c, and its depth through
    the reference's draw kernels (which do not read the maps): bit-exact."""
    sc, fr, maps = border_frame()
    rd = O.RefDraw(sc, VIEW)
    for k in range(len(sc.shadows)):
        rc, m = rd.shadow_map(k)
        assert rc == 0
        assert np.array_equal(m.view(np.uint32), maps[k].view(np.uint32)), k
    rd.clear_zbuffer()
    assert rd.draw_all() == 0
    db = rd.get_frame()[3]
    assert np.array_equal(db.view(np.uint32), fr.db.view(np.uint32))


def expected_fmip(pts, uv, bias, nmip):
    """av_draw_normmap_mip.c:37-45 evaluated in float64: the largest
    |dUV| / (edge length in pixels)^2 over the three edges, then
    clamp(|log2 dt| / 2 + mipBias, 0, numMip - 1).  Small triangles (integer
    bounding box under 96 pixels, trisetup.c) use their truncated vertices,
    as the small path does (Templates.py:230-231); large ones the float
    vertices of the tiled path."""
    p = np.asarray(pts, np.float64)
    small = max(np.ptp(np.trunc(p), axis=0)) < 96
    if small:
        p = np.trunc(p)
    u = np.asarray(uv, np.float64)
    dt = 0.0
    for i, j in ((0, 1), (0, 2), (1, 2)):
        d2 = float(((p[j] - p[i]) ** 2).sum())
        dt = max(dt, *np.abs((u[j] - u[i]) / d2))
    return min(max(abs(np.log2(dt)) / 2 + bias, 0.0), nmip - 1.0), small


def test_trilinear_level_selection():
    """The per-triangle mip level on the oracle against the formula, read
    back from constant-per-level textures: a mid-range level and the upper
    clamp on the tiled path; the lower clamp, dt > 1 and truncated vertices
    on the small path."""
    sc, view, cases = kat.mip_scene()
    fr = O.Frame(view.w, view.h)
    O.clear_depth(fr.db)
    O.draw_all(sc, view, fr, [])
    nmip = int(np.log2(kat.MIP_SIDE))
    paths = []
    for k, (pts, uv, bias) in enumerate(cases):
        px = fr.tri_id == k
        assert px.sum() >= 20, k
        got = fr.ro[px].astype(np.float64) / kat.MIP_LEVEL_VALUE - 1.0
        want, small = expected_fmip(pts, uv, bias, nmip)
        paths.append(small)
        assert np.abs(got - want).max() <= 2e-3, (k, float(got.min()), float(got.max()), want)
    assert paths == [False, False, True, True, True]
    # the clamps are reached, and case 4 tells truncated edges from float ones
    assert expected_fmip(*cases[1], nmip)[0] == nmip - 1 and expected_fmip(*cases[2], nmip)[0] == 0.0
    pts, uv, bias = cases[4]
    p, u = np.asarray(pts), np.asarray(uv, np.float64)
    dt_float = max(max(np.abs((u[j] - u[i]) / ((p[j] - p[i]) ** 2).sum())) for i, j in ((0, 1), (0, 2), (1, 2)))
    float_level = abs(np.log2(dt_float)) / 2 + bias
    got4 = fr.ro[fr.tri_id == 4].astype(np.float64) / kat.MIP_LEVEL_VALUE - 1.0
    assert np.abs(got4 - float_level).min() > 5e-3
