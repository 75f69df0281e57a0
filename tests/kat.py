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


# shadow-map border taps (av_alpha_max.c:53-84: a cascade counts its five
# taps only when the centre tap lies in [2, 2 wS - 2) on both axes)
BORDER_T0 = 20000            # the receivers' constant texel
BORDER_CASCADES = [((0.0, 0.0, 0.0), 22.1), ((1.5, 1.0, 0.0), 22.1)]   # (centre, texels per unit), 64^2 each
BORDER_DEPTH = 10.0          # receiver plane z; the cascades sit at z = -20 looking down +z
BORDER_SMALL_DEPTH = 9.9     # the small receivers, just in front of the plane
BORDER_SMALL_OFFSET = (0.3, 0.2)   # the small receivers' vertices sit this far past whole pixels


def shadow_border_scene(w=96, h=72):
    """A receiver plane at z = 10 facing the camera and lit head-on, a caster
    behind the camera (rejected by the view, drawn into the maps) over the
    half-plane x + y < 0, and two 64^2 cascades looking down +z that each
    end inside the view: cascade 0 holds |x|, |y| <= 1.45 around the axis,
    cascade 1 the same around (1.5, 1.0).  Where cascade 0's centre tap
    falls on its two outer rows or columns, the caster lies under it and
    cascade 1 does not reach, so the count there must be 0.  The texture is
    constant and the vertex light 0: a pixel's red value is
    T0 * light * 1.6 with light = (s * amb + 5 - s) / 5, from which the
    shadow count s reads back.

    Receivers: two large triangles at z = 10 (the tiled path, rows
    < 16 * (h // 16)) and, at z = 9.9 in front of them, 8 x 8-pixel small
    ones over the bottom 16 rows (the only receivers of rows 64-71) and over
    the left half of rows 40-55, where the shadow and cascade 0's border
    reach them too."""
    rng = np.random.default_rng(12)
    z = BORDER_DEPTH
    T = lambda pts: tri(w, h, pts)
    big = [T([(-30.0, -20.0, z), (130.0, 10.0, z), (10.0, 110.0, z)]),
           T([(130.0, -20.0, z), (130.0, 110.0, z), (-30.0, 110.0, z)])]
    small = []
    zs = BORDER_SMALL_DEPTH
    cells = [(cx, cy) for cy in range(h - 16, h, 8) for cx in range(0, w, 8)]
    cells += [(cx, cy) for cy in range(h - 32, h - 16, 8) for cx in range(0, w // 2, 8)]
    for cx, cy in cells:
        x0, y0 = cx + BORDER_SMALL_OFFSET[0], cy + BORDER_SMALL_OFFSET[1]
        small.append(T([(x0, y0, zs), (x0 + 8, y0, zs), (x0, y0 + 8, zs)]))
        small.append(T([(x0 + 8, y0, zs), (x0 + 8, y0 + 8, zs), (x0, y0 + 8, zs)]))
    caster = [[(-5.0, 5.0, -5.0), (5.0, -5.0, -5.0), (-5.0, -5.0, -5.0)]]
    plane = np.full(16 * 16, BORDER_T0, np.uint16)

    def group(tris, flags, normal):
        xyz = np.asarray(tris, np.float32).reshape(-1, 3)
        n = xyz.shape[0]
        vn = np.tile(np.asarray(normal, np.float32), (n, 1))
        uv = rng.random((n, 2)).astype(np.float32)
        return S.Group(xyz, uv, vn, np.zeros((n, 3), np.float32), (plane, plane.copy(), plane.copy()), 16, flags)

    groups = [group(big, S.SHADOW, (0, 0, -1)), group(small, S.SHADOW, (0, 0, -1)), group(caster, 0, (0, 0, 1))]
    cams = [S.ShadowCam.facing(64, s, c, (0.0, 0.0), dist=20.0) for c, s in BORDER_CASCADES]
    return S.Scene(groups, [], np.asarray(S.LIGHT_INTS[0], np.float32), np.array([0, 0, -1], np.float32), 0.2, cams)


def border_counts(sc, maps, tri_id, w, h):
    """The shadow count av_alpha_max.c gives each pixel of the receiver plane
    of shadow_border_scene, from the maps, with `clear` False where a tap
    coordinate lies within 0.02 texels of an integer (where the float
    rounding of the interpolated position decides); and the mask of pixels
    whose cascade-0 centre tap is outside [2, 62) on a map texel that the
    caster covers while cascade 1 is out of reach (count 0 by the border
    rule alone).

    A pixel's world position is the point of its receiver under the
    pixel's corner, except that on the small receivers it is the point under
    the corner plus BORDER_SMALL_OFFSET: the small path truncates vertex
    screen positions (Templates.py:230-231) while the interpolated position
    runs between the true vertices."""
    ys, xs = np.mgrid[0:h, 0:w].astype(np.float64)
    n0 = sc.groups[0].ntris
    small = (tri_id >= n0) & (tri_id < n0 + sc.groups[1].ntris)
    xs = xs + np.where(small, BORDER_SMALL_OFFSET[0], 0.0)
    ys = ys + np.where(small, BORDER_SMALL_OFFSET[1], 0.0)
    Z = np.where(small, BORDER_SMALL_DEPTH, BORDER_DEPTH)
    X = (xs - w // 2) * Z / SCALE
    Y = (ys - h // 2) * Z / SCALE
    total = np.zeros((h, w), np.int64)
    clear = np.ones((h, w), bool)
    exposed = np.ones((h, w), bool)
    for k, cam in enumerate(sc.shadows):
        m = maps[k]
        ws = cam.dim // 2
        depth = Z - float(cam.pos[2])
        fx = -(X - float(cam.pos[0])) * cam.scale
        fy = (Y - float(cam.pos[1])) * cam.scale
        for f in (fx, fy):
            frac = np.abs(f - np.round(f))
            clear &= frac > 0.02
        sx = np.trunc(fx).astype(np.int64) + ws
        sy = np.trunc(fy).astype(np.int64) + ws
        inside = (sx >= 2) & (sx < 2 * ws - 2) & (sy >= 2) & (sy < 2 * ws - 2)
        cnt = np.zeros((h, w), np.int64)
        for dy, dx in ((0, 0), (2, 0), (-2, 0), (0, 2), (0, -2)):
            ty = np.clip(sy + dy, 0, 2 * ws - 1)
            tx = np.clip(sx + dx, 0, 2 * ws - 1)
            cnt += inside & (m[ty, tx] < depth)
        total += cnt
        onmap = (sx >= 0) & (sx < 2 * ws) & (sy >= 0) & (sy < 2 * ws)
        under = onmap & (m[np.clip(sy, 0, 2 * ws - 1), np.clip(sx, 0, 2 * ws - 1)] < depth)
        exposed &= (~inside & under) if k == 0 else ~inside
    return np.minimum(total, 5), clear, exposed


def decode_shadow_count(red, amb=0.2):
    """The shadow count s of shadow_border_scene's receivers from the red
    plane (T0 * light * LInt.x, light = (s * amb + 5 - s) * 0.2)."""
    light = red.astype(np.float64) / (BORDER_T0 * float(S.LIGHT_INTS[0][0]))
    return np.rint((1.0 - light) / ((1.0 - amb) * 0.2)).astype(np.int64)


# trilinear mip selection (av_draw_normmap_mip.c:37-45): the per-triangle
# level fmip = clamp(|log2 dt| / 2 + mipBias, 0, numMip - 1) from the
# largest |dUV| / (edge length in pixels)^2 over the three edges
MIP_SIDE = 16                # levels of side 1, 2, 4, 8, 16 (numMip = 4), smallest first
MIP_LEVEL_VALUE = 1000       # level k holds MIP_LEVEL_VALUE * (k + 1) in every texel


def mip_scene(w=192, h=144):
    """One triangle per group, each a case of the level selection, at depth
    5 and apart on screen: (screen vertices, uvs, mipBias).  Every level of
    the texture is a constant, the vertex light is 1 and the normals face
    away from the light, so a pixel's red value is
    MIP_LEVEL_VALUE * (1 + fmip): the level blend reads back as fmip.
      0 tiled path, mid-range level (dt = 2^-5: fmip 2.5)
      1 tiled path, dt tiny: clamped to numMip - 1
      2 small path, mipBias -10: clamped to 0
      3 small path, dt > 1 (a 6-pixel triangle spanning 100 texture units)
      4 small path, fractional vertices (edge lengths from the truncated ones)
    """
    cases = [([(4.0, 4.0), (120.0, 4.0), (4.0, 70.0)], [(0, 0), (242.0, 0), (0, 100.0)], 0.0),
             ([(70.0, 140.0), (190.0, 140.0), (190.0, 76.0)], [(0, 0), (0.01, 0), (0, 0.01)], 0.0),
             ([(130.25, 10.25), (160.25, 10.25), (130.25, 40.25)], [(0, 0), (3.0, 0), (0, 3.0)], -10.0),
             ([(10.25, 100.25), (16.25, 100.25), (10.25, 106.25)], [(0, 0), (100.0, 0), (0, 100.0)], 0.0),
             ([(30.7, 90.2), (60.4, 91.9), (35.5, 120.8)], [(0, 0), (150.0, 1.0), (10.0, 20.0)], 0.3)]
    nmip = int(np.log2(MIP_SIDE))
    chain = np.concatenate([np.full(4 ** k, MIP_LEVEL_VALUE * (k + 1), np.uint16) for k in range(nmip + 1)])
    groups = []
    for pts, uv, bias in cases:
        xyz = np.asarray(tri(w, h, [(x, y, 5.0) for x, y in pts]), np.float32)
        groups.append(S.Group(xyz, np.asarray(uv, np.float32), np.tile(np.float32([0, 0, 1]), (3, 1)),
                              np.ones((3, 3), np.float32), (chain, chain.copy(), chain.copy()), nmip, S.MIP,
                              mip_bias=bias))
    sc = S.Scene(groups, [], np.asarray(S.LIGHT_INTS[0], np.float32), np.array([0, 0, -1], np.float32), 0.2, [])
    return sc, view(w, h), cases
