"""The tiled shadow depth pass against the per-caster pass and the oracle.

CLDraw.shadowMap (Ops.py:1089-1141: trisetupOrtho.c, drawmin.c,
drawminalpha.c) draws the casters binned to 32 x 32-texel tiles, each tile's
minimum taken in shared memory and texels a span cannot lower skipped before
the exact depth.  Every map here must equal the oracle's (drawmin.c run
serially) and the per-caster pass's bit for bit: maps whose side is not a
multiple of the tile, casters that cover many tiles (rows replayed to each
tile's first row), alpha-tested casters, passes into an uncleared map, and a
unit queue too small for the pass (the same launch then draws per caster,
and the queue grows for the next pass).
"""
import os

import numpy as np
import pytest

import oracle as O
from axi_visualizer_b200 import scenes as S
from axi_visualizer_b200.ops import SceneRenderer

pytestmark = pytest.mark.gpu


def _maps(sc, mode, passes=1, cast_masks=None):
    R = SceneRenderer(sc, 64, 48, device=0)
    R.draw.setShadowMode(mode)
    out = []
    for k in range(len(sc.shadows)):
        R.draw.clearShadowMap(k)
        for p in range(passes):
            cast = cast_masks[p] if cast_masks else [g.cast for g in sc.groups]
            R.draw.shadowMap(k, cast, R.shaders, sc.bias)
        out.append(R.draw.getSHM(k).copy())
    R.draw.sync()
    return out


def _oracle(sc, passes=1, cast_masks=None):
    out = []
    for k, s in enumerate(sc.shadows):
        m = O.new_shadow_map(s.dim)
        for p in range(passes):
            O.shadow_map(sc, k, m, cast=cast_masks[p] if cast_masks else None)
        out.append(m)
    return out


def _same(a, b, what):
    assert a.shape == b.shape
    d = int((a.view(np.uint32) != b.view(np.uint32)).sum())
    assert d == 0, f"{what}: {d} texels differ"


def _check(sc, **kw):
    want = _oracle(sc, **kw)
    tiled = _maps(sc, 1, **kw)
    tiled_sorted = _maps(sc, 2, **kw)
    per_caster = _maps(sc, 0, **kw)
    for k in range(len(sc.shadows)):
        _same(tiled[k], want[k], f"tiled map {k} vs oracle")
        _same(tiled_sorted[k], want[k], f"tiled (front first) map {k} vs oracle")
        _same(per_caster[k], want[k], f"per-caster map {k} vs oracle")
        assert (want[k] < 65535).any(), "the map has casters"


@pytest.mark.parametrize("seed", [3, 11])
def test_tiled_maps_equal_oracle(seed):
    _check(S.scene_small(seed=seed))


def test_map_sides_not_multiple_of_tile():
    sc = S.scene_small(seed=5)
    sc.shadows = [S.ShadowCam.facing(200, 200 / 2 / 30.0, (0, 0, 0), S.SUN),
                  S.ShadowCam.facing(45, 45 / 2 / 25.0, (1, 0, 2), S.SUN)]
    _check(sc)


def test_casters_over_many_tiles():
    """A coarse terrain whose triangles span hundreds of texels: every tile of
    a caster replays its rows up to the tile's first row."""
    rng = np.random.default_rng(21)
    xyz, vn, uv = S.terrain(rng, 6, 8.0, (-24.0, 0.0, -24.0), 3.0)
    rgb, _ = S.noise_texture(rng, 32)
    sx, sn, su = S.icospheres(rng, 6, 2.0, 6.0, -15, 15)
    groups = [S._group(xyz, vn, uv, rgb, S.SHADOW, 0.2), S._group(sx, sn, su, rgb, S.SHADOW, 0.2)]
    shadows = [S.ShadowCam.facing(777, 777 / 2 / 30.0, (0, 0, 0), S.SUN),
               S.ShadowCam.facing(512, 512 / 2 / 12.0, (3, 0, -2), S.SUN)]
    _check(S._finish(groups, [], shadows))


def test_uncleared_map_takes_the_minimum_of_passes():
    sc = S.scene_small(seed=7)
    masks = [[True, False, False], [False, True, True]]
    _check(sc, passes=2, cast_masks=masks)


def test_unit_queue_overflow_draws_per_caster_then_grows():
    """A unit queue of 7 entries (AXR_SHADOW_UNIT_QUEUE, read when a map's
    first tiled pass allocates it): the first passes overflow and are drawn
    per caster in the same launches, the queue grows, and the later passes
    are tiled; every map equals the oracle's."""
    sc = S.scene_small(seed=4)
    want = _oracle(sc)
    R = SceneRenderer(sc, 64, 48, device=0)
    R.draw.setShadowMode(2)
    os.environ["AXR_SHADOW_UNIT_QUEUE"] = "7"
    try:
        for k in range(len(sc.shadows)):
            R.draw.clearShadowMap(k)
            R.draw.shadowMap(k, [g.cast for g in sc.groups], R.shaders, sc.bias)
    finally:
        del os.environ["AXR_SHADOW_UNIT_QUEUE"]
    R.draw.sync()
    assert all(r[0] > 0 for r in R.draw.shadowOverflows()), "the first passes overflowed"
    for k in range(len(sc.shadows)):
        _same(R.draw.getSHM(k), want[k], f"overflowed pass, map {k}")
    for rep in range(2):    # tiled after the growth
        for k in range(len(sc.shadows)):
            R.draw.clearShadowMap(k)
            R.draw.shadowMap(k, [g.cast for g in sc.groups], R.shaders, sc.bias)
        R.draw.sync()
        for k in range(len(sc.shadows)):
            _same(R.draw.getSHM(k), want[k], f"pass {rep} after growth, map {k}")
    assert all(r[0] == 1 for r in R.draw.shadowOverflows()), "no overflow after the growth"
