"""Known-answer edge-case scenes, built in screen space.

The camera sits at the origin looking down +z with basis rows
[view (0,0,1), horizontal (-1,0,0), vertical (0,1,0)], so trisetup.c maps a
point (X, Y, Z) to screen (W/2 + s X/Z, H/2 + s Y/Z).  `tri(...)` places a
vertex near a requested screen position at a requested depth.  Each case is
a list of groups of triangles; the reference has no tests, so these cases
are authored to reach the corners of its arithmetic.
"""
import numpy as np

from axi_visualizer_b200 import scenes as S

SCALE = 200.0


def view(w, h):
    vv = np.array([[0, 0, 1], [-1, 0, 0], [0, 1, 0]], np.float32)
    return S.View(w, h, np.zeros(3, np.float32), vv, float(np.float32(SCALE)), 50.0, 50.0)


def vert(w, h, sx, sy, z):
    return ((sx - w // 2) * z / SCALE, (sy - h // 2) * z / SCALE, z)


def tri(w, h, pts):
    """pts: three (screen x, screen y, depth) tuples."""
    return [vert(w, h, *p) for p in pts]


def _group(tris, rng, flags=0, tex=16, alpha_index=0, uv=None):
    xyz = np.asarray(tris, np.float64).reshape(-1, 3)
    n = len(tris)
    vn = np.tile(np.array([0, 0, 1.0]), (3 * n, 1))
    if uv is None:
        uv = rng.random((3 * n, 2))
    rgb, _ = S.noise_texture(rng, tex)
    return S._group(xyz, vn, np.asarray(uv), rgb, flags, 0.2, alpha_index=alpha_index)


def case_scenes(w=96, h=72):
    """{name: (scene, view)} for the edge cases."""
    rng = np.random.default_rng(11)
    out = {}
    T = lambda pts: tri(w, h, pts)

    # triangles with vertices on and across tile borders, small and large
    border = [T([(15.5, 3.2, 5), (16.0, 20.7, 6), (31.99, 16.0, 7)]),
              T([(32.0, 32.0, 4), (47.9, 32.0, 4), (40.0, 47.99, 4)]),
              T([(0.0, 0.0, 9), (95.9, 0.5, 9), (48.0, 71.9, 9)]),
              T([(-30.0, -20.0, 8), (130.0, 10.0, 8), (10.0, 110.0, 8)])]
    out["tile_borders"] = [border]

    # flat bottom / flat top (equal projected y), small and large
    flat = [T([(10.0, 10.0, 5), (30.0, 10.0, 6), (20.0, 25.0, 7)]),
            T([(40.0, 40.0, 5), (60.0, 55.0, 5), (80.0, 55.0, 5)]),
            T([(2.0, 5.0, 6), (90.0, 5.0, 6), (50.0, 70.0, 6)]),
            T([(5.0, 2.0, 7), (50.0, 66.0, 7), (93.0, 66.0, 7)])]
    out["flat_edges"] = [flat]

    # slivers, duplicate vertices, zero-height rows, a point
    sliv = [T([(10.2, 10.1, 5), (10.4, 10.3, 5), (10.3, 10.9, 5)]),   # same integer bbox: rejected
            T([(20.0, 20.0, 5), (20.0, 20.0, 5), (30.0, 22.0, 5)]),
            T([(40.0, 30.0, 5), (70.0, 31.0, 5), (41.0, 30.2, 5)]),
            T([(50.0, 50.0, 5), (50.5, 70.0, 5), (51.0, 50.0, 5)])]
    out["slivers"] = [sliv]

    # crossing the near plane or behind the camera: rejected whole
    near = [[(0.1, 0.1, 5.0), (1.0, 0.2, -1.0), (0.2, 1.0, 5.0)],
            [(0.1, 0.1, -5.0), (1.0, 0.2, -1.0), (0.2, 1.0, -5.0)],
            T([(20.0, 20.0, 5), (60.0, 25.0, 5), (30.0, 60.0, 5)])]
    out["near_plane"] = [near]

    # exact depth ties: the same triangle twice in a group, again in a later
    # group, and a large copy (large pass comes after the small pass)
    a = T([(20.0, 15.0, 5), (50.0, 20.0, 5), (30.0, 50.0, 5)])
    big = T([(0.0, 0.0, 5), (95.0, 2.0, 5), (40.0, 71.0, 5)])
    out["depth_ties"] = [[a, a, big], [a, big, a]]

    # 200 large triangles stacked over one tile (overflows the reference's
    # 128-entry bins; unbounded here)
    stack = [T([(-10.0 + 0.01 * k, 1.0, 5 + 0.01 * k), (100.0, 3.0 + 0.05 * k, 5), (10.0, 70.0, 6)]) for k in range(200)]
    out["bin_overflow"] = [stack]

    # masked and empty groups
    out["masked_empty"] = [[], border, flat]      # group 1 is masked out

    # alpha test: a checkerboard mask sampled at texel corners and centres
    quads = []
    for k in range(6):
        x0, y0 = 4 + 15 * k, 8 + 9 * k
        quads.append(T([(x0, y0, 5), (x0 + 14, y0, 5), (x0, y0 + 40, 5)]))
    out["alpha_edges"] = [quads]
    scenes = {}
    for name, groups in out.items():
        gs = []
        for gi, tris in enumerate(groups):
            if name == "alpha_edges":
                uv = np.tile(np.array([[0.0, 0.0], [0.5, 0.0], [0.0, 0.5]]), (len(tris), 1))
                g = _group(tris, rng, S.ALPHA, tex=16, uv=uv)
            else:
                g = _group(tris, rng, S.CULL if gi == 1 and name == "depth_ties" else 0) if tris else None
            if g is None:
                g = _group([T([(1.0, 1.0, 5), (2.0, 1.0, 5), (1.0, 2.0, 5)])], rng)
                g = S.Group(g.xyz[:0], g.uv[:0], g.vn[:0], g.li[:0], g.tex, g.tex_size, 0)
            gs.append(g)
        alphas = []
        if name == "alpha_edges":
            m = (np.indices((16, 16)).sum(0) % 2).astype(np.uint8)
            alphas = [(m.reshape(-1), 16)]
        sc = S.Scene(gs, alphas, np.asarray(S.LIGHT_INTS[0], np.float32), S.LIGHT_DIRS[0].astype(np.float32), 0.2,
                     [S.ShadowCam.facing(64, 64 / 2 / 12.0, (0, 0, 6), (0.0, 0.0), dist=20.0)])
        scenes[name] = sc
    return scenes, view(w, h)


def masks(name, ngroups):
    return [0, 1] + [0] * (ngroups - 2) if name == "masked_empty" else None
