"""The vertex stage (PyOpenCL27C/Pipe/vert.c: transform, Ttranslate, vertL)
in the oracle, pinned to the reference: the golden fixture made by the
reference's own kernels (tests/golden/make_golden.py, ref_vertex.npz), and --
where oracle/_ref is built -- the reference kernels run live.  Bit-exact."""
import hashlib
import os
import sys

import numpy as np
import pytest

import oracle as O
from axi_visualizer_b200 import scenes as S

GOLD = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLD)
import make_golden as MG  # noqa: E402  (vertex_ops: the fixture's inputs)

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def same(a, b):
    return a.shape == b.shape and np.array_equal(np.asarray(a, np.float32).view(np.uint32),
                                                 np.asarray(b, np.float32).view(np.uint32))


def apply_ops(sc, ops, L):
    """The fixture's operations on the oracle, in place on the scene's arrays."""
    for kind, g, a, b, args in ops:
        G = sc.groups[g]
        if kind == "rotate":
            O.transform(G.xyz, G.vn, args[0], args[1], args[2], a, b)
        else:
            O.translate(G.xyz, args[0], a, b)
    for g, on in enumerate(L["mask"]):
        if on:
            G = sc.groups[g]
            G.li[...] = O.vert_light(G.xyz, G.vn, L["dir_int"], L["dir_dir"], L["amb"], L["point_int"],
                                     L["point_pos"], L["spot_int"], L["spot_dir"], L["spot_pos"])


def test_vertex_stage_equals_reference_golden():
    gold = np.load(os.path.join(GOLD, "ref_vertex.npz"))
    seed, (w, h, pos), ops, L = MG.vertex_ops()
    sc = S.scene_small(seed=seed, flags=0, with_alpha=True)
    before = [g.xyz.copy() for g in sc.groups]
    apply_ops(sc, ops, L)
    for g, G in enumerate(sc.groups):
        assert same(G.xyz, gold[f"g{g}_xyz"]), g
        assert same(G.vn, gold[f"g{g}_vn"]), g
        assert same(G.li, gold[f"g{g}_li"]), g
    # the operations moved what they name and nothing else
    assert not np.array_equal(sc.groups[1].xyz[37:5001], before[1][37:5001])
    assert np.array_equal(sc.groups[1].xyz[:37], before[1][:37])
    assert np.array_equal(sc.groups[1].xyz[5001:], before[1][5001:])
    assert np.array_equal(sc.groups[0].xyz[:5], before[0][:5])
    fr, smaps = O.render(sc, S.default_view(w, h, pos=pos))
    for k, m in enumerate(smaps):
        assert sha(m) == str(gold[f"shm{k}_sha256"])
    for n, a in (("r", fr.ro), ("g", fr.go), ("b", fr.bo), ("db", fr.db)):
        assert sha(a) == str(gold[f"{n}_sha256"]), n


def test_vert_light_formula_cases():
    """Hand-computed vertL cases.  Only lights 1.. add (light 0 is shaded
    per pixel).  A point or spot light adds where dot(normal, x - light) > 0,
    a spot light also where dot(direction, x - light) > 0.  The ambient floor
    applies per channel."""
    f = np.float32
    xyz = np.zeros((3, 3), f)
    vn = np.array([[0, 1, 0], [0, -1, 0], [1, 0, 0]], f)
    dirs_i = np.array([[9, 9, 9], [1, 0, 0]], f)
    dirs_d = np.array([[0, 1, 0], [0, 1, 0]], f)
    li = O.vert_light(xyz, vn, dirs_i, dirs_d, 0.1)
    assert li[0, 0] == f(f(f(1.0) + f(0.5)) * f(0.66)) and li[0, 1] == f(0.1)
    assert li[1, 0] == f(0.1)                        # max(0, -1 + 0.5) = 0
    assert li[2, 0] == f(f(0.5) * f(0.66))
    # point light at (0, -2, 0): x - light = (0, 2, 0) faces normal +y only
    li = O.vert_light(xyz, vn, dirs_i[:1], dirs_d[:1], 0.0, point_int=[[5, 5, 5]], point_pos=[[0, -2, 0]])
    assert li[0, 0] == f(f(f(1.0) / f(f(1.0) + f(2.0) * f(2.0))) * f(5))
    assert li[1].tolist() == [0, 0, 0] and li[2].tolist() == [0, 0, 0]
    # spot light at (0, 3, 0): x - light = (0, -3, 0) faces normal -y
    spot = dict(spot_int=[[2, 2, 2]], spot_pos=[[0, 3, 0]])
    lit = f(f(f(f(1.0) * f(1.0)) / f(f(1.5) + f(3.0) * f(3.0))) * f(2))
    li = O.vert_light(xyz, vn, dirs_i[:1], dirs_d[:1], 0.0, spot_dir=[[0, -1, 0]], **spot)
    assert li[1, 0] == lit and li[0, 0] == 0 and li[2, 0] == 0
    # the same light pointing up (away from the vertices) adds nothing
    li = O.vert_light(xyz, vn, dirs_i[:1], dirs_d[:1], 0.0, spot_dir=[[0, 1, 0]], **spot)
    assert not li.any()


def test_transform_identity_and_inverse():
    rng = np.random.default_rng(3)
    xyz = rng.standard_normal((100, 3)).astype(np.float32)
    vn = rng.standard_normal((100, 3)).astype(np.float32)
    x0, n0 = xyz.copy(), vn.copy()
    O.transform(xyz, vn, np.eye(3), np.eye(3), (0, 0, 0), 0, 100)
    assert np.array_equal(xyz, x0) and np.array_equal(vn, n0)
    r = MG.rot_mat(0.4, -1.2, 2.0)
    O.transform(xyz, vn, np.eye(3), r, (1, 2, 3), 10, 90)
    assert np.array_equal(xyz[:10], x0[:10]) and np.array_equal(xyz[90:], x0[90:])
    assert np.allclose(xyz[10:90], ((x0[10:90] - (1, 2, 3)) @ r) + (1, 2, 3), atol=1e-5)
    assert np.allclose(vn[10:90], n0[10:90] @ r, atol=1e-5)
    O.translate(xyz, (1, -1, 0.5), 0, 100)
    assert np.allclose(xyz[:10], x0[:10] + (1, -1, 0.5), atol=1e-6)


@needs_ref
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_vertex_stage_equals_reference_kernels_live(seed):
    """Random sub-ranges, rotations and light sets (including no extra
    lights, only the primary directional light, and many point/spot lights)
    through the reference's own kernels and through the oracle."""
    rng = np.random.default_rng(100 + seed)
    sc = S.scene_small(seed=seed, flags=0, with_alpha=True)
    view = S.default_view(64, 48)
    rd = O.RefDraw(sc, view)
    for _ in range(6):
        g = int(rng.integers(0, len(sc.groups)))
        nv = sc.groups[g].ntris * 3
        a = int(rng.integers(0, nv))
        b = int(rng.integers(a, nv + 1))
        if rng.random() < 0.6:
            old = MG.rot_mat(*rng.uniform(-3, 3, 3))
            new = MG.rot_mat(*rng.uniform(-3, 3, 3))
            o = rng.uniform(-5, 5, 3)
            assert rd.rotate(old, new, o, a, b, g) == 0
            O.transform(sc.groups[g].xyz, sc.groups[g].vn, old, new, o, a, b)
        else:
            c = rng.uniform(-5, 5, 3)
            assert rd.translate(c, a, b, g) == 0
            O.translate(sc.groups[g].xyz, c, a, b)
    for nd, npt, nsp in ((3, 0, 0), (1, 0, 0), (2, 5, 7), (4, 40, 0), (1, 0, 33)):
        di = rng.uniform(0, 2, (nd, 3)).astype(np.float32)
        dd = rng.standard_normal((nd, 3)).astype(np.float32)
        pi = rng.uniform(0, 3, (npt, 3)).astype(np.float32)
        pp = rng.uniform(-10, 10, (npt, 3)).astype(np.float32)
        si = rng.uniform(0, 3, (nsp, 3)).astype(np.float32)
        sd = rng.standard_normal((nsp, 3)).astype(np.float32)
        sp = rng.uniform(-10, 10, (nsp, 3)).astype(np.float32)
        amb = float(rng.uniform(0, 0.5))
        mask = [1] * len(sc.groups)
        assert rd.vert_light(mask, di, dd, amb, pi, pp, si, sd, sp) == 0
        for g, G in enumerate(sc.groups):
            xyz, vn, li = rd.geometry(g)
            assert same(xyz, G.xyz) and same(vn, G.vn), g
            want = O.vert_light(G.xyz, G.vn, di, dd, amb, pi, pp, si, sd, sp)
            assert same(li, want), (g, nd, npt, nsp)
