"""Post/ssao.c, Post/dof.c and the bloom (Post/blur.c + blur2.c) in the
oracle, pinned to the reference: golden
digests made by the reference's own kernels (tests/golden/ref_post.npz) and,
where oracle/_ref is built, the kernels run live.  Bit-exact."""
import hashlib
import os
import sys

import numpy as np
import pytest

import oracle as O
from axi_visualizer_b200 import scenes as S

GOLD = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLD)
import make_golden as MG  # noqa: E402

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("i", range(len(MG.POST_CASES)))
def test_post_effects_equal_reference_golden(i):
    gold = np.load(os.path.join(GOLD, "ref_post.npz"))
    seed, w, h, pos = MG.POST_CASES[i]
    sc = S.scene_small(seed=seed, flags=0, with_alpha=True)
    view = S.default_view(w, h, pos=pos)
    fr, _ = O.render(sc, view)
    before = fr.ro.copy()
    O.ssao(fr, view.sscale, MG.post_rand())
    assert sha(np.stack((fr.ro, fr.go, fr.bo))) == str(gold[f"p{i}_ssao_sha256"])
    assert (fr.ro != before).mean() > 0.05          # the occlusion darkened part of the frame
    for f in MG.POST_FOCUS:
        O.dof(fr, f)
        assert sha(np.stack((fr.ro, fr.go, fr.bo))) == str(gold[f"p{i}_dof{f:g}_sha256"]), f
    O.bloom(fr)
    assert sha(np.stack((fr.ro, fr.go, fr.bo))) == str(gold[f"p{i}_bloom_sha256"])


@needs_ref
@pytest.mark.parametrize("seed", [0, 4])
@pytest.mark.parametrize("size", [(160, 128), (176, 90)])
def test_post_effects_equal_reference_kernels_live(seed, size):
    w, h = size
    rnd = np.random.default_rng(seed).random(48).astype(np.float32)
    sc = S.scene_small(seed=seed, flags=0, with_alpha=True)
    view = S.default_view(w, h, pos=(2, 5, -14))
    fr, _ = O.render(sc, view)
    rd = O.RefDraw(sc, view)
    rd.clear_zbuffer()
    assert rd.draw_all() == 0
    rd.ssao(rnd)
    O.ssao(fr, view.sscale, rnd)
    r, g, b, _ = rd.get_frame()
    assert np.array_equal(r, fr.ro) and np.array_equal(g, fr.go) and np.array_equal(b, fr.bo)
    for f in (1.5, 12.0, 40.0):
        rd.dof(f)
        O.dof(fr, f)
        r, g, b, _ = rd.get_frame()
        assert np.array_equal(r, fr.ro) and np.array_equal(g, fr.go) and np.array_equal(b, fr.bo), f
    before = fr.ro.copy()
    rd.bloom()
    O.bloom(fr)
    r, g, b, _ = rd.get_frame()
    assert np.array_equal(r, fr.ro) and np.array_equal(g, fr.go) and np.array_equal(b, fr.bo), "bloom"
    assert (fr.ro != before).mean() > 0.3


def test_dof_leaves_rows_below_the_region():
    sc = S.scene_small(seed=2)
    view = S.default_view(128, 100, pos=(-20, 3, 5))
    fr, _ = O.render(sc, view)
    before = fr.ro.copy()
    O.dof(fr, 2.0)
    assert np.array_equal(fr.ro[96:], before[96:])
    assert not np.array_equal(fr.ro[:96], before[:96])
