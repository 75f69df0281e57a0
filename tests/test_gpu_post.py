"""CLDraw.ssao / dof / blur on the device (k_ssao, k_dof and the k_bloom_*
passes through the C ABI) against the oracle on the same frame: bit-exact
colour planes.  The frame is set from the oracle's own render, so the
comparison is of the post effects alone; depth is left untouched by both."""
import numpy as np
import pytest

import oracle as O
from axi_visualizer_b200 import scenes as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("size", [(160, 128), (192, 101), (320, 240)])
@pytest.mark.parametrize("seed", [1, 3])
def test_ssao_dof_match_oracle(size, seed):
    from axi_visualizer_b200.ops import SceneRenderer
    w, h = size
    sc = S.scene_small(seed=seed)
    view = S.default_view(w, h, pos=(2, 5, -14))
    fr, _ = O.render(sc, view)
    R = SceneRenderer(sc, w, h)
    d = R.draw
    R.set_view(view)
    rnd = np.random.default_rng(seed).random(48).astype(np.float32)
    d.setFrame(fr.ro, fr.go, fr.bo, fr.db)
    d.ssao(rnd)
    O.ssao(fr, view.sscale, rnd)
    r, g, b, db = [x.copy() for x in d.getFrame()]
    assert np.array_equal(db.view(np.uint32), fr.db.view(np.uint32))
    assert np.array_equal(r, fr.ro) and np.array_equal(g, fr.go) and np.array_equal(b, fr.bo), "ssao"
    for f in (1.5, 8.0, 30.0):
        d.dof(f)
        O.dof(fr, f)
        r, g, b, _ = [x.copy() for x in d.getFrame()]
        assert np.array_equal(r, fr.ro) and np.array_equal(g, fr.go) and np.array_equal(b, fr.bo), f"dof {f}"
    for rep in range(2):                       # the bloom twice: its planes keep no state between calls
        d.blur()
        O.bloom(fr)
        r, g, b, _ = [x.copy() for x in d.getFrame()]
        assert np.array_equal(r, fr.ro) and np.array_equal(g, fr.go) and np.array_equal(b, fr.bo), f"bloom {rep}"


def test_ssao_default_table_and_errors():
    from axi_visualizer_b200.ops import SceneRenderer
    from axi_visualizer_b200._lib import AxrError
    sc = S.scene_small(seed=2)
    R = SceneRenderer(sc, 64, 48)
    R.frame(S.default_view(64, 48))
    R.draw.ssao()                              # draws its table once, as the reference does
    t = R.draw._ssao_rand.copy()
    R.draw.ssao()
    assert np.array_equal(t, R.draw._ssao_rand)
    with pytest.raises(AxrError):
        R.draw.ssao(np.zeros(16, np.float32))
