"""Host-side logic without a GPU: scenes, cameras, material parsing, mip
layout, the correctly rounded log2 shared by oracle and kernels."""
import math
import struct

import numpy as np
import pytest

import oracle as O
from axi_visualizer_b200 import scenes as S


def test_named_scene_sizes():
    assert S.scene_c1().ntris == 24192
    sc = S.scene_c2()
    assert sc.ntris == 1044288
    assert [g.ntris for g in sc.groups] == [262144, 262144, 240000, 240000, 40000]
    assert [s.dim for s in sc.shadows] == [2048, 2048]
    assert sc.alphas[0][1] == 1024 and 0.55 < sc.alphas[0][0].mean() < 0.65


def test_frame_bytes_formula():
    """The roofline's per-frame algorithmic bytes for the 1080p scene:
    132 T + sum over cascades (36 T_cast + 24 T_alpha_cast) + 10 W H +
    4 sum S^2, about 269 MB (texture and shadow-map reads excluded)."""
    import bench
    sc = S.scene_c2()
    T = sc.ntris
    assert all(g.cast for g in sc.groups)
    want = 132 * T + 2 * (36 * T + 24 * 40000) + 10 * 1920 * 1080 + 4 * 2 * 2048 * 2048
    assert (bench.W, bench.H) == (1920, 1080)
    assert bench.frame_bytes(sc) == want
    assert 268e6 < want < 270e6


def test_issue_roofline():
    """The instruction-issue roofline: issued warp instructions per launch
    (from the ncu capture) / launch time, against SMs x 4 schedulers x the
    sampled SM clock; kernels without a captured count get none."""
    import bench
    n = bench.NCU_ISSUED["k_shadow_raster"]
    r = bench.issue_of("k_shadow_raster", 250e-6, 148, 1965.0)
    assert r["warp_inst_per_launch"] == n
    assert r["peak_winst_per_s"] == 148 * 4 * 1965e6
    assert abs(r["frac"] - n / 250e-6 / (148 * 4 * 1965e6)) < 1e-12
    assert 0.5 < r["frac"] < 1.0
    assert bench.issue_of("k_clear_shadow", 10e-6, 148, 1965.0) is None
    roof = bench.roofline_of("k_shade", {"k_shade": (2.0, 10)}, {"k_shade": 50e6}, 6500.0, "measured", 10)
    assert abs(roof["avg_us"] - 200.0) < 1e-9 and abs(roof["achieved"] - 250.0) < 1e-9
    assert roof["traffic"] == bench.NCU_TRAFFIC["k_shade"] and roof["issue"]["frac"] > 0


def test_camera_bases_orthonormal():
    for a, b in ((0.3, 0.2), (1.7 * math.pi, 0.52), (-2.0, -0.7)):
        for m in (S.camera_basis(a, b), S.view_mat(a, b)):
            assert np.allclose(m @ m.T, np.eye(3), atol=1e-12)
    v = S.default_view(1920, 1080)
    assert abs(v.sscale - 960 / math.tan(35 * math.pi / 180)) < 1e-3


def test_material_flags():
    assert S.flags_from_string("mip shadow  cull") == S.MIP | S.SHADOW | S.CULL
    assert S.flags_from_string("alpha ") == S.ALPHA
    assert S.flags_from_string({"alpha": 1, "shadow": 1}) == S.ALPHA | S.SHADOW
    assert S.flags_from_string("") == 0


def test_cldraw_material_args_without_gpu():
    from axi_visualizer_b200.ops import CLDraw

    class Fake:
        gSize = [3, 3, 3]
    flags, aidx = CLDraw._material_args(Fake(), {0: "mip shadow", 1: {"alpha": 2}, 2: "cull"})
    assert flags.tolist() == [S.MIP | S.SHADOW, S.ALPHA, S.CULL] and aidx.tolist() == [0, 2, 0]
    with pytest.raises(Exception):
        CLDraw._material_args(Fake(), ["mip"])


def test_mip_bias_per_draw_as_the_reference_passes_it():
    """A group's mipBias for one drawAll: np.float32(material["mip"]) when
    its material is the normal-mapped mip dict ("normal" and "mip",
    Ops.py:687, 797-799), else the setMipBias value (0 until set).  In other
    materials "mip" is only a flag, so {"alpha": a, "mip": 1} renders at bias
    0, and a string material after a dict one does not keep the dict's bias.
    The library is told only when a group's bias changes."""
    from axi_visualizer_b200.ops import CLDraw
    calls = []

    class FakeLib:
        def axr_draw_all(self, *a):
            calls.append(("draw",))
            return 0

        def axr_set_mip_bias(self, h, tn, b):
            calls.append(("bias", tn, float(b.value)))
            return 0

        def axr_set_normal_material(self, h, tn, m, r, metal):
            calls.append(("normal", tn, m, float(r.value), metal))
            return 0

    class Fake:
        gSize = [3, 3, 3, 3]
        SHADOWMAP = {}
        NM = {0: 7}
        _h = None
        _L = FakeLib()
        _material_args = CLDraw._material_args
        _dict_mip_biases = staticmethod(CLDraw._dict_mip_biases)
        _draw_mip_biases = CLDraw._draw_mip_biases
        _draw_normal_materials = CLDraw._draw_normal_materials
        _apply_mip_bias = CLDraw._apply_mip_bias
        setMipBias = CLDraw.setMipBias

    f = Fake()
    f._normal = {}
    f._mip_bias = [np.float32(0)] * 4
    f._set_bias = [np.float32(0)] * 4
    shaders = ["mip shadow", {"alpha": 0, "mip": 1}, {"normal": (0, 1.0), "roughness": 0, "mip": 0.5},
               {"alpha": 0}]
    CLDraw.drawAll(f, shaders, shadowIds=[])
    assert calls == [("bias", 2, 0.5), ("normal", 2, 7, 1.0, 0), ("draw",)]
    calls.clear()
    CLDraw.drawAll(f, shaders, shadowIds=[])          # unchanged: no library call
    assert calls == [("draw",)]
    calls.clear()
    CLDraw.drawAll(f, ["mip", "mip", "mip", "mip"], shadowIds=[])   # per draw: the dict's bias is gone
    assert calls == [("bias", 2, 0.0), ("draw",)]
    calls.clear()
    CLDraw.setMipBias(f, 1, 2.0)
    assert calls == [("bias", 1, 2.0)]
    calls.clear()
    CLDraw.drawAll(f, ["mip", {"alpha": 0, "mip": 1}, "mip", "mip"], shadowIds=[])   # the set value holds
    assert calls == [("draw",)]
    assert [float(b) for b in f._mip_bias] == [0.0, 2.0, 0.0, 0.0]


def test_scene_renderer_hands_every_group_field_to_the_draw(monkeypatch):
    """SceneRenderer passes each field of a scene group that the oracle
    reads (positions, uvs, normals, vertex light, texture planes and mip
    chain, flags, alpha index, mipBias) and each cascade to the draw
    runtime.  Recorded through a stand-in CLDraw, without a GPU."""
    import kat
    from axi_visualizer_b200 import ops
    log = []

    class Rec:
        def __init__(self, *a, **k):
            pass

        def __getattr__(self, name):
            return lambda *a, **k: log.append((name, a, k))

    real = ops.CLDraw
    monkeypatch.setattr(ops, "CLDraw", Rec)
    sc, view, cases = kat.mip_scene()
    sc.groups[1].flags |= S.ALPHA
    sc.alphas = [(np.ones(kat.MIP_SIDE ** 2, np.uint8), kat.MIP_SIDE)]
    sc.shadows = [S.ShadowCam.facing(64, 3.0, (0, 0, 6), (0.0, 0.0), dist=20.0)]
    R = ops.SceneRenderer(sc, view.w, view.h)
    adds = [a for n, a, k in log if n == "addTextureGroup"]
    mips = [k.get("mip") for n, a, k in log if n == "addTextureGroup"]
    assert len(adds) == len(sc.groups)
    for g, a, mip in zip(sc.groups, adds, mips):
        for got, want in zip(a, (g.xyz, g.uv, g.vn) + tuple(g.tex)):
            assert np.array_equal(got, want)
        assert mip == 1 << g.tex_size
    lis = {a[0]: a[1] for n, a, k in log if n == "setVertLight"}
    assert all(np.array_equal(lis[i], g.li) for i, g in enumerate(sc.groups))
    biases = {a[0]: float(a[1]) for n, a, k in log if n == "setMipBias"}
    assert biases == {i: float(g.mip_bias) for i, g in enumerate(sc.groups) if g.mip_bias}
    assert [n for n, a, k in log].count("addTexAlpha") == 1
    assert [a[:2] for n, a, k in log if n == "addShadowMap"] == [(0, 64)]
    assert [a[0] for n, a, k in log if n == "placeShadowMapBasis"] == [0]
    # materials: flags and alpha index as the oracle reads them; the mipBias
    # goes through setMipBias only (no dict bias)
    fake = type("F", (), {"gSize": [3] * len(sc.groups)})()
    flags, aidx = real._material_args(fake, R.shaders)
    assert flags.tolist() == [g.flags for g in sc.groups]
    assert aidx.tolist() == [g.alpha_index for g in sc.groups]
    assert real._dict_mip_biases(R.shaders, len(sc.groups)) == {}


# every method of the reference's CLDraw (PyOpenCL27C/Ops.py:127-1230)
REFERENCE_CLDRAW_METHODS = """
__init__ addBoneWeights addNrmMap addOpacityMap addRghMap addShadowMap addTexAlpha addTexture addTextureGroup
blur blurTest boneTransform clearShadowMap clearShadowOpMap clearZBuffer copyTo dof drawAll drawDirectional
exposure gamma genVoxels getArgs getBoneWeights getBuffers getFrame getGIM getSHM getShadow getVertNorms
getVertPoints getVoxels highlight initBoneOrigin initBoneTransforms invbt mipShadowMap placeShadowMap rotate
setBoneTransform setHostSkyTex setPos setPrimaryLight setReflTex setScaleCull setSkyTex setVM setupWave
shadowMap ssao tonemap translate updateWave vertLight voxCopy voxLight voxTerrain
""".split()


def test_every_reference_cldraw_method_is_provided_or_refused():
    """A caller of the reference class finds each method: implemented, or
    raising NotImplementedError with the reason (no AttributeError)."""
    from axi_visualizer_b200.ops import CLDraw
    d = CLDraw.__new__(CLDraw)          # no handle: only attribute lookup is exercised
    provided, refused = [], []
    for name in REFERENCE_CLDRAW_METHODS:
        if name in CLDraw.__dict__:
            assert callable(CLDraw.__dict__[name]), name
            provided.append(name)
            continue
        with pytest.raises(NotImplementedError):
            getattr(d, name)
        refused.append(name)
    assert {"drawAll", "shadowMap", "getFrame", "vertLight", "rotate", "getVertPoints"} <= set(provided)
    assert "voxLight" in refused and "getBuffers" in refused
    with pytest.raises(AttributeError):
        getattr(d, "noSuchMethod")


def test_vertex_getters_use_the_padded_layout():
    """getVertPoints / getVertNorms return the reference's align34 layout
    (Ops.py:124-125, 290-297): (T, 3, 4) float32 with a zero fourth
    component."""
    from axi_visualizer_b200.ops import CLDraw, _pad4
    v = np.arange(18, dtype=np.float32).reshape(6, 3)
    out = _pad4(v)
    assert out.shape == (2, 3, 4) and out.dtype == np.float32
    assert np.array_equal(out[..., :3].reshape(-1, 3), v) and not out[..., 3].any()

    class Fake:
        def getVertices(self, tn):
            return v + tn, -v, np.zeros_like(v)
    assert np.array_equal(CLDraw.getVertPoints(Fake(), 1)[..., :3].reshape(-1, 3), v + 1)
    assert np.array_equal(CLDraw.getVertNorms(Fake(), 0)[..., :3].reshape(-1, 3), -v)


def test_mip_chain_layout():
    rgb = np.random.default_rng(0).integers(0, 8000, (16, 16, 3))
    planes, num = S.texture_planes(rgb.astype(np.uint16), True)
    assert num == 4 and planes[0].size == (4 * 16 * 16 - 1) // 3
    assert np.array_equal(planes[0][-256:], rgb[..., 0].reshape(-1))        # largest level last
    lvl1 = (rgb[0::2, 0::2] + rgb[1::2, 0::2] + rgb[0::2, 1::2] + rgb[1::2, 1::2]) >> 2
    start = (8 * 8 - 1) // 3                                              # levels 1x1, 2x2, 4x4 come first
    assert np.array_equal(planes[0][start:start + 64], lvl1[..., 0].reshape(-1))


def f32(x):
    return struct.unpack("f", struct.pack("f", x))[0]


def test_log2_correctly_rounded():
    L = O.lib()
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.random(20000) * 10.0 ** rng.integers(-30, 30, 20000),
                         np.array([1.0, 2.0, 0.5, 1e-40, 3.4e38, 1.5, 1.4142135])]).astype(np.float32)
    bad = 0
    for x in xs:
        got = L.orc_log2f(float(x))
        want = f32(math.log2(float(x)))
        if got != want:
            bad += 1
            # differs only where the exact value sits on a float rounding boundary
            assert abs(got - want) <= abs(want) * 2 ** -23 + 1e-45
    assert bad <= 2
    assert L.orc_log2f(0.0) == -math.inf and L.orc_log2f(math.inf) == math.inf
    assert math.isnan(L.orc_log2f(-1.0))


def test_vert_light_matches_formula():
    vn = np.array([[0, -1, 0], [0.6, -0.8, 0]], np.float32)
    li = S.vert_light(vn, S.LIGHT_DIRS, S.LIGHT_INTS, 0.2)
    d1 = S.LIGHT_DIRS[1].astype(np.float32)
    s = max(0.0, float(np.float32(vn[0] @ d1)) + 0.5) * 0.66
    assert abs(li[0, 0] - max(0.2, s * 0.5 + max(0.0, float(vn[0] @ S.LIGHT_DIRS[2]) + 0.5) * 0.66 * 0.1)) < 1e-5
    assert (li >= 0.2).all()


def test_stress_scene_composition():
    """The stress scene's layout at a reduced size: 12 terrain bands + 4
    sphere groups, one texture each, alpha-tested bands 2, 5, 8 and sphere
    groups 0, 2 against one mask of the texture side; the full size has
    2 * 2048^2 + 80 * 20000 = 9,988,608 triangles, 29.0% alpha-tested."""
    sc = S.scene_c5(terrain_n=64, spheres=400, tex=64)
    assert len(sc.groups) == 16
    assert sc.ntris == 2 * 64 * 64 + 80 * 400
    alpha = [k for k, g in enumerate(sc.groups) if g.flags & S.ALPHA]
    assert alpha == [2, 5, 8, 12, 14]
    assert all(g.flags & S.MIP and g.tex_size == 6 for g in sc.groups)
    assert sc.alphas[0][1] == 64 and sc.alphas[0][0].size == 64 * 64
    full_alpha = (3 * 2 * 2048 * 2048 // 12 + 2 * 20000 * 80 // 4) / (2 * 2048 * 2048 + 80 * 20000)
    assert abs(full_alpha - 0.29) < 0.001
