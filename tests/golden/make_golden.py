"""Generates the golden fixtures in this directory from the reference itself.

Run in a checkout where the reference is present (it is read, never copied):

    python oracle/build_ref.py                 # reference kernels -> oracle/_ref
    python tests/golden/make_golden.py

1. ref_frames.npz: frames and shadow maps rendered by the reference's own
   OpenCL kernels compiled for the CPU (oracle/_ref, run work-item by
   work-item) on small seeded scenes; colour planes and depth are stored
   whole, plus SHA-256 digests of every array.
2. ref_terrain.npz: vertex positions and UVs of the reference's own
   VertTerrain.create (PyOpenCL27C/VertObjects.py:643-700) for a 4x4 height
   field, and Utils.createMips (PyOpenCL27C/Utils.py:79-93) of an 8x8 RGB
   texture, imported from the reference with a stub for its unused numexpr
   import.
4. ref_multi.npz: frames of the 4-way blend terrain material rendered by
   the reference's own PyOpenCL27C/Shaders/drawmulti.c (oracle/_ref) on the
   seeded scenes of MULTI_CASES (reference-kernel variant: the other groups
   bilinear at their base level, no shadow lookup); SHA-256 digests.
5. ref_post.npz: Post/ssao.c, Post/dof.c and the bloom of Post/blur.c +
   blur2.c of the reference (oracle/_ref) applied to the frames of
   POST_CASES (ssao with the table post_rand(), dof at each focus of
   POST_FOCUS, then the bloom); SHA-256 digests of the colour planes after
   each step.
3. ref_vertex.npz: the vertex stage through the reference's own
   PyOpenCL27C/Pipe/vert.c kernels (oracle/_ref): a rotation about an origin
   and a translation of vertex sub-ranges, then per-vertex light from
   directional, point and spot lights, on a small seeded scene; the inputs
   (vertex_ops()), the resulting vertex arrays, and digests of the shadow
   maps and the frame rendered from them.
"""
import hashlib
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
REF = os.environ.get("AXR_REFERENCE", "/root/reference")

CASES = [  # (seed, width, height, camera position)
    (3, 160, 120, (0, 8, -30)),
    (1, 160, 128, (3, 2, -8)),
    (2, 128, 96, (-20, 3, 5)),
]


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def frames():
    import oracle as O
    from axi_visualizer_b200 import scenes as S
    out = {}
    for i, (seed, w, h, pos) in enumerate(CASES):
        sc = S.scene_small(seed=seed, flags=0, with_alpha=True)
        view = S.default_view(w, h, pos=pos)
        rd = O.RefDraw(sc, view)
        for k in range(len(sc.shadows)):
            rc, m = rd.shadow_map(k)
            assert rc == 0
            out[f"c{i}_shm{k}"] = m
        rd.clear_zbuffer()
        assert rd.draw_all() == 0
        r, g, b, db = rd.get_frame()
        out.update({f"c{i}_r": r, f"c{i}_g": g, f"c{i}_b": b, f"c{i}_db": db})
    # the full-size 1080p scene (reference-kernel variant): digests only
    sc = S.reference_kernel_variant(S.scene_c2())
    view = S.default_view(1920, 1080)
    rd = O.RefDraw(sc, view)
    for k in range(len(sc.shadows)):
        rc, m = rd.shadow_map(k, nthreads=1)
        out[f"hd_shm{k}_sha256"] = np.array(digest(m))
    rd.clear_zbuffer()
    assert rd.draw_all() == 0
    r, g, b, db = rd.get_frame()
    for n, a in (("r", r), ("g", g), ("b", b), ("db", db)):
        out[f"hd_{n}_sha256"] = np.array(digest(a))
    for k in list(out):
        if not k.endswith("sha256"):
            out[k + "_sha256"] = np.array(digest(out[k]))
    np.savez_compressed(os.path.join(HERE, "ref_frames.npz"), **out)


MULTI_CASES = [  # (seed, width, height, camera position, target)
    (9, 192, 144, (0, 30, -40), (0, 12, 0)),
    (10, 192, 144, (5, 20, -20), (0, 12, 0)),
    (9, 160, 128, (-10, 8, -12), (0, 12, 0)),
]


def multi():
    import oracle as O
    from axi_visualizer_b200 import scenes as S
    out = {}
    for i, (seed, w, h, pos, target) in enumerate(MULTI_CASES):
        sc = S.reference_kernel_variant(S.scene_multi(seed=seed))
        rd = O.RefDraw(sc, S.default_view(w, h, pos=pos, target=target))
        rd.clear_zbuffer()
        assert rd.draw_all() == 0
        for n, a in zip(("r", "g", "b", "db"), rd.get_frame()):
            out[f"m{i}_{n}_sha256"] = np.array(digest(a))
    np.savez_compressed(os.path.join(HERE, "ref_multi.npz"), **out)


POST_CASES = [  # (seed, width, height, camera position); 128 and 144 are multiples of 16
    (3, 160, 128, (0, 8, -30)),
    (1, 192, 144, (3, 2, -8)),
    (2, 128, 100, (-20, 3, 5)),
]
POST_FOCUS = (2.0, 8.0, 20.0)


def post_rand():
    return np.random.default_rng(44).random(48).astype(np.float32)


def post():
    import oracle as O
    from axi_visualizer_b200 import scenes as S
    out = {}
    rnd = post_rand()
    for i, (seed, w, h, pos) in enumerate(POST_CASES):
        sc = S.scene_small(seed=seed, flags=0, with_alpha=True)
        rd = O.RefDraw(sc, S.default_view(w, h, pos=pos))
        rd.clear_zbuffer()
        assert rd.draw_all() == 0
        rd.ssao(rnd)
        r, g, b, _ = rd.get_frame()
        out[f"p{i}_ssao_sha256"] = np.array(digest(np.stack((r, g, b))))
        for f in POST_FOCUS:
            rd.dof(f)
            r, g, b, _ = rd.get_frame()
            out[f"p{i}_dof{f:g}_sha256"] = np.array(digest(np.stack((r, g, b))))
        rd.bloom()
        r, g, b, _ = rd.get_frame()
        out[f"p{i}_bloom_sha256"] = np.array(digest(np.stack((r, g, b))))
    np.savez_compressed(os.path.join(HERE, "ref_post.npz"), **out)


def rot_mat(a, b, c):
    """VertObject.rotate (PyOpenCL27C/VertObjects.py:281-294): rotX @ rotZ @ rotY."""
    ca, sa, cb, sb, cc, sc = np.cos(a), np.sin(a), np.cos(b), np.sin(b), np.cos(c), np.sin(c)
    rx = np.array([[1, 0, 0], [0, ca, -sa], [0, sa, ca]])
    ry = np.array([[cb, 0, sb], [0, 1, 0], [-sb, 0, cb]])
    rz = np.array([[cc, -sc, 0], [sc, cc, 0], [0, 0, 1]])
    return rx @ rz @ ry


def vertex_ops():
    """Inputs of the vertex-stage fixture: the scene, the operations in
    order, the lights.  Shared by the generator and the tests."""
    r1 = rot_mat(0.3, 1.1, -0.4)
    r2 = rot_mat(-0.7, 0.2, 0.9)
    ops = [
        # (kind, group, start vertex, end vertex, args)
        ("rotate", 1, 37, 5001, (np.eye(3), r1, (1.5, 0.25, -2.0))),
        ("rotate", 1, 37, 5001, (r1.T, r2, (1.5, 0.25, -2.0))),
        ("translate", 0, 5, 1530, ((0.75, -0.5, 1.25),)),
        ("rotate", 2, 0, 240, (np.eye(3), r1, (0.0, 0.0, 0.0))),
    ]
    lights = dict(
        dir_int=np.array([(1.6, 1.4, 1.2), (0.5, 0.5, 0.5), (0.1, 0.2, 0.6)], np.float32),
        dir_dir=np.array([(0.3, -0.8, 0.5), (-0.3, 0.8, -0.5), (0.0, 1.0, 0.0)], np.float32),
        point_int=np.array([(3.0, 2.0, 1.0), (0.5, 1.5, 4.0)], np.float32),
        point_pos=np.array([(2.0, 3.0, -1.0), (-6.0, 1.0, 4.0)], np.float32),
        spot_int=np.array([(2.0, 2.0, 2.0), (1.0, 0.2, 0.2)], np.float32),
        spot_dir=np.array([(0.0, -1.0, 0.0), (0.6, -0.8, 0.0)], np.float32),
        spot_pos=np.array([(0.0, 6.0, 0.0), (-5.0, 4.0, -3.0)], np.float32),
        amb=0.2, mask=(1, 1, 0))
    return 3, (192, 144, (3, 4, -14)), ops, lights


def vertex():
    import oracle as O
    from axi_visualizer_b200 import scenes as S
    seed, (w, h, pos), ops, L = vertex_ops()
    sc = S.scene_small(seed=seed, flags=0, with_alpha=True)
    view = S.default_view(w, h, pos=pos)
    rd = O.RefDraw(sc, view)
    for kind, g, a, b, args in ops:
        rc = rd.rotate(args[0], args[1], args[2], a, b, g) if kind == "rotate" else rd.translate(args[0], a, b, g)
        assert rc == 0
    assert rd.vert_light(L["mask"], L["dir_int"], L["dir_dir"], L["amb"], L["point_int"], L["point_pos"],
                         L["spot_int"], L["spot_dir"], L["spot_pos"]) == 0
    out = {}
    for g in range(len(sc.groups)):
        xyz, vn, li = rd.geometry(g)
        out.update({f"g{g}_xyz": xyz, f"g{g}_vn": vn, f"g{g}_li": li})
    for k in range(len(sc.shadows)):
        rc, m = rd.shadow_map(k)
        assert rc == 0
        out[f"shm{k}_sha256"] = np.array(digest(m))
    rd.clear_zbuffer()
    assert rd.draw_all() == 0
    for n, a in zip(("r", "g", "b", "db"), rd.get_frame()):
        out[f"{n}_sha256"] = np.array(digest(a))
    np.savez_compressed(os.path.join(HERE, "ref_vertex.npz"), **out)


def terrain():
    sys.modules.setdefault("numexpr", types.ModuleType("numexpr"))
    sys.path.insert(0, os.path.join(REF, "PyOpenCL27C"))
    from Utils import createMips
    from VertObjects import VertTerrain

    class Viewer:
        def __init__(self):
            self.vtNames, self.vtextures, self.vertpoints, self.vertnorms = {}, [], [], []
            self.vertu, self.vertv, self.vertBones, self.matShaders = [], [], [], {}
            self.texAlphas, self.vaNames = [], {}

    rng = np.random.default_rng(7)
    hts = rng.standard_normal((5, 5)) * 2
    v = Viewer()
    t = VertTerrain(v, [-2, 0, -2], heights=hts.copy(), texture=os.path.join(REF, "Assets", "Grass1.png"), uvspread=2)
    t.created()
    pts = np.array(v.vertpoints[0]).reshape(-1, 3)
    u = np.array(v.vertu[0]).reshape(-1)
    vv = np.array(v.vertv[0]).reshape(-1)
    tex = rng.integers(0, 8000, (8, 8, 3))
    mips = createMips(tex)
    np.savez_compressed(os.path.join(HERE, "ref_terrain.npz"), heights=hts, xyz=pts, u=u, v=vv, tex=tex, mips=mips)


if __name__ == "__main__":
    frames()
    terrain()
    vertex()
    multi()
    post()
    print("golden fixtures written to", HERE)
