"""Seeded synthetic scenes in the reference's data layout.

Everything here is host-side input preparation (numpy, float32 outputs):
triangle soups with per-vertex positions, normals, UVs and light `I`,
textures preprocessed like the reference, full mip chains, alpha masks,
cameras and shadow cameras.  No benchmark data is read: the configurations
are seeded stand-ins with the shapes and value distributions of the
rasterizer's named workloads (terrain + icospheres + alpha quads).

Conventions follow the reference:
  - terrain triangulation and UVs of VertTerrain.create
    (PyOpenCL27C/VertObjects.py:643-700), UV wrap of texMode "repeat"
    (:193-195); quads split like VertPlane (:743-756)
  - normals point along the view ray on visible faces (the direction
    trisetup_cull.c:52 keeps), i.e. inward on closed meshes, -y on terrain
  - texture texels `c*c/8` as uint16 (VertObjects.py:123-131), mip chain
    smallest level first (Utils.createMips, PyOpenCL27C/Utils.py:79-93)
  - alpha mask `floor(a/255 + 0.4)` (VertObjects.py:96-100)
  - camera basis of Compute.viewVec/vVhorz/vVvert/lookAt
    (PyOpenCL27C/Compute.py:271-274,465-479), shadow basis Utils.viewMat
    (PyOpenCL27C/Utils.py:14-20), scale/cull from Compute.py:127-133
  - per-vertex light `I` of vert.vertL (PyOpenCL27C/Pipe/vert.c:38-87)
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

MIP, ALPHA, SHADOW, CULL, MULTI, NORMAL = 1, 2, 4, 8, 16, 32


def flags_from_string(s) -> int:
    """Material string (or dict) -> flag bits, as Ops.drawAll tests substrings."""
    if isinstance(s, dict):
        keys = " ".join(str(k) for k in s.keys())
    else:
        keys = str(s)
    f = 0
    if "mip" in keys:
        f |= MIP
    if "alpha" in keys:
        f |= ALPHA
    if "shadow" in keys:
        f |= SHADOW
    if "cull" in keys:
        f |= CULL
    if "multi" in keys:
        f |= MULTI
    if "normal" in keys:
        f |= NORMAL
    return f


# ---------------------------------------------------------------- cameras

def view_vec(a: float, b: float) -> np.ndarray:
    return np.array([math.sin(a) * math.cos(b), -math.sin(b), math.cos(a) * math.cos(b)])


def view_mat(a: float, b: float) -> np.ndarray:
    a2, b2 = a + math.pi / 2, b - math.pi / 2
    return np.array([[math.sin(a) * math.cos(b), -math.sin(b), math.cos(a) * math.cos(b)],
                     [-math.sin(a2), 0.0, -math.cos(a2)],
                     [-math.sin(a) * math.cos(b2), math.sin(b2), -math.cos(a) * math.cos(b2)]])


def look_at(pos, target):
    d = np.asarray(target, float) - np.asarray(pos, float)
    a = math.pi / 2 - math.atan2(d[2], d[0])
    b = -math.atan2(d[1], math.sqrt(d[0] ** 2 + d[2] ** 2))
    return a, b


def camera_basis(a: float, b: float) -> np.ndarray:
    """[viewVec, vVhorz, vVvert] of Compute.py:312-314,465-479."""
    vv = view_vec(a, b)
    a2 = a + math.pi / 2
    horz = -np.array([math.sin(a2), 0.0, math.cos(a2)])
    b2 = b - math.pi / 2
    vert = -np.array([math.sin(a) * math.cos(b2), -math.sin(b2), math.cos(a) * math.cos(b2)])
    return np.stack((vv, horz, vert))


@dataclass
class View:
    w: int
    h: int
    pos: np.ndarray          # (3,) float32
    vv: np.ndarray           # (3,3) float32
    sscale: float
    cax: float
    cay: float

    @staticmethod
    def perspective(w, h, pos, target=None, fov_deg=70.0, angles=None):
        w2, h2 = int(w / 2), int(h / 2)
        scale = w2 / math.tan(fov_deg * math.pi / 360)
        cax = w2 / scale + 2
        cay = h2 / scale + 2
        if angles is None:
            angles = look_at(pos, target if target is not None else (0, 0, 0))
        vv = camera_basis(*angles)
        return View(w, h, np.asarray(pos, np.float32), vv.astype(np.float32),
                    float(np.float32(scale)), float(np.float32(cax)), float(np.float32(cay)))


@dataclass
class ShadowCam:
    dim: int
    scale: float
    pos: np.ndarray
    vv: np.ndarray

    @staticmethod
    def facing(dim, scale, centre, light_angles, dist=120.0):
        vv = view_mat(*light_angles)
        pos = np.asarray(centre, float) - vv[0] * dist
        return ShadowCam(dim, float(np.float32(scale)), pos.astype(np.float32), vv.astype(np.float32))


# ---------------------------------------------------------------- geometry

@dataclass
class Group:
    xyz: np.ndarray          # (V,3) float32, V = 3T
    uv: np.ndarray           # (V,2) float32
    vn: np.ndarray           # (V,3) float32
    li: np.ndarray           # (V,3) float32
    tex: tuple               # (r, g, b) uint16 flat planes
    tex_size: int            # lenT, or numMip for mip materials
    flags: int
    alpha_index: int = 0
    mip_bias: float = 0.0
    cast: bool = True
    # normal-mapped materials: RGBA bytes, one texel per texel of the texture
    # (or chain); the "normal" pair's second value (roughness); metal
    nm: np.ndarray = None
    roughness: float = 0.5
    metal: bool = False

    @property
    def ntris(self) -> int:
        return self.xyz.shape[0] // 3


@dataclass
class Scene:
    groups: list
    alphas: list = field(default_factory=list)   # list of (mask uint8 [N*N], N)
    lint: np.ndarray = None
    ldir: np.ndarray = None
    amb: float = 0.2
    shadows: list = field(default_factory=list)  # ShadowCam
    bias: float = 0.2

    @property
    def ntris(self) -> int:
        return sum(g.ntris for g in self.groups)


def terrain(rng, n, cell, origin, height_sd, uvspread=2.0):
    """(n x n)-cell heightfield of N(0,1)*height_sd heights."""
    h = (rng.standard_normal((n + 1, n + 1)) * height_sd).astype(np.float64)
    return terrain_from_heights(h, cell, origin, uvspread)


def terrain_from_heights(h, cell, origin, uvspread=2.0):
    """VertTerrain.create triangulation of an (n+1)x(n+1) height field, per-cell
    UVs wrapped to [0,1) (texMode "repeat"), -y facing normals from central
    differences."""
    h = np.asarray(h, np.float64)
    n = h.shape[0] - 1
    i = np.arange(n + 1, dtype=np.float64)
    X = origin[0] + i[:, None] * cell + 0 * i[None, :]
    Z = origin[2] + i[None, :] * cell + 0 * i[:, None]
    P = np.stack((X, h + origin[1], Z), axis=-1)                 # (n+1,n+1,3)
    gx = np.gradient(h, cell, axis=0)
    gz = np.gradient(h, cell, axis=1)
    N = np.stack((gx, -np.ones_like(h), gz), axis=-1)
    N /= np.linalg.norm(N, axis=-1, keepdims=True)
    ii, jj = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    ii = ii.reshape(-1)
    jj = jj.reshape(-1)
    # triangle A: (i,j) (i+1,j) (i,j+1); triangle B: (i+1,j+1) (i,j+1) (i+1,j)
    ia = np.stack((ii, ii + 1, ii), 1)
    ja = np.stack((jj, jj, jj + 1), 1)
    ib = np.stack((ii + 1, ii, ii + 1), 1)
    jb = np.stack((jj + 1, jj + 1, jj), 1)
    ti = np.stack((ia, ib), 1).reshape(-1, 3)                    # cell-major A,B
    tj = np.stack((ja, jb), 1).reshape(-1, 3)
    xyz = P[ti, tj].reshape(-1, 3)
    vn = N[ti, tj].reshape(-1, 3)
    uA = np.stack((ii, ii + 0.99, ii), 1)
    vA = np.stack((jj, jj, jj + 0.99), 1)
    uB = np.stack((ii + 0.99, ii, ii + 0.99), 1)
    vB = np.stack((jj + 0.99, jj + 0.99, jj), 1)
    u = np.stack((uA, uB), 1).reshape(-1) / uvspread
    v = np.stack((vA, vB), 1).reshape(-1) / uvspread
    uv = np.stack((u % 1, v % 1), 1)
    return xyz, vn, uv


_ICO = None


def _icosphere80():
    global _ICO
    if _ICO is None:
        t = (1 + 5 ** 0.5) / 2
        v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                      [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], float)
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
             (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
        tris = []
        for a, b, c in f:
            A, B, C = v[a], v[b], v[c]
            ab = (A + B); ab /= np.linalg.norm(ab)
            bc = (B + C); bc /= np.linalg.norm(bc)
            ca = (C + A); ca /= np.linalg.norm(ca)
            tris += [(A, ab, ca), (B, bc, ab), (C, ca, bc), (ab, bc, ca)]
        _ICO = np.array(tris)                                     # (80,3,3) unit sphere
    return _ICO


def icospheres(rng, count, rmin, rmax, lo, hi):
    base = _icosphere80()
    r = rng.uniform(rmin, rmax, count)
    c = rng.uniform(lo, hi, (count, 3))
    P = base[None] * r[:, None, None, None] + c[:, None, None, :]
    Nrm = -np.broadcast_to(base[None], P.shape)                  # inward
    d = base.reshape(-1, 3)
    u = np.arctan2(d[:, 2], d[:, 0]) / (2 * np.pi) + 0.5
    v = np.arcsin(np.clip(d[:, 1], -1, 1)) / np.pi + 0.5
    uv = np.broadcast_to(np.stack((u, v), 1)[None], (count, d.shape[0], 2))
    return P.reshape(-1, 3), Nrm.reshape(-1, 3), uv.reshape(-1, 2)


def quads(rng, count, lo, hi, smin, smax, ground=0.0):
    """Upright two-triangle quads (VertPlane n=1 split and UVs)."""
    s = rng.uniform(smin, smax, count)
    yaw = rng.uniform(0, 2 * np.pi, count)
    cx = rng.uniform(lo, hi, count)
    cz = rng.uniform(lo, hi, count)
    h1 = np.stack((np.cos(yaw), np.zeros(count), np.sin(yaw)), 1) * s[:, None]
    h2 = np.stack((np.zeros(count), np.ones(count), np.zeros(count)), 1) * s[:, None]
    c = np.stack((cx, np.full(count, ground), cz), 1) - h1 / 2
    n = np.cross(h1, h2)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    n = -n
    t1 = np.stack((c, c + h2, c + h1), 1)
    t2 = np.stack((c + h1 + h2, c + h1, c + h2), 1)
    P = np.stack((t1, t2), 1).reshape(-1, 3)
    Nn = np.repeat(n, 6, axis=0)
    uv1 = np.array([(0, 0), (0, 1), (1, 0)], float)
    uv2 = np.array([(1, 1), (1, 0), (0, 1)], float)
    uv = np.broadcast_to(np.stack((uv1, uv2))[None], (count, 2, 3, 2)).reshape(-1, 2)
    return P, Nn, uv * 0.999


# ---------------------------------------------------------------- textures

def noise_texture(rng, n, alpha_p=None):
    """n x n RGBA8 uniform noise -> preprocessed planes (c*c/8 as uint16).
    Returns (rgb uint16 (n,n,3), alpha mask uint8 (n,n) or None)."""
    rgba = rng.integers(0, 256, (n, n, 4)).astype(np.float64)
    if alpha_p is not None:
        rgba[..., 3] = np.where(rng.random((n, n)) < alpha_p, 255.0, 0.0)
    ta = rgba * rgba / 8.0
    rgb = ta[..., :3].astype(np.uint16)
    mask = None
    if alpha_p is not None:
        mask = np.floor(rgba[..., 3] / 255 + 0.4).astype(np.uint8)
    return rgb, mask


def create_mips(rgb):
    """Integer 2x2 box mip chain, smallest level first, as (texels, 3) int."""
    a = rgb.astype(np.int64)
    levels = [a]
    for _ in range(int(math.log2(rgb.shape[0]))):
        b = a[:-1:2] + a[1::2]
        a = (b[:, :-1:2] + b[:, 1::2]) >> 2
        levels.append(a)
    levels.reverse()
    return np.concatenate([x.reshape(-1, 3) for x in levels], axis=0)


def normal_map(rng, n, mip: bool):
    """Seeded bumpy tangent-space normal map of side n as RGBA bytes (the
    layout CLDraw.addNrmMap stores; A = 0), full resolution or a create_mips
    chain smallest level first."""
    h = rng.standard_normal((n + 1, n + 1))
    gx, gy = h[:-1, 1:] - h[:-1, :-1], h[1:, :-1] - h[:-1, :-1]
    v = np.stack([-gx, -gy, np.full_like(gx, 2.0)], axis=-1)
    v /= np.linalg.norm(v, axis=-1, keepdims=True)
    rgb = np.clip(np.round((v * 0.5 + 0.5) * 255.0), 0, 255).astype(np.int64)
    flat = create_mips(rgb) if mip else rgb.reshape(-1, 3)
    out = np.zeros((flat.shape[0], 4), np.uint8)
    out[:, :3] = flat
    return out.reshape(-1)


def texture_planes(rgb, mip: bool):
    if mip:
        t = create_mips(rgb).astype(np.uint16)
        planes = (np.ascontiguousarray(t[:, 0]), np.ascontiguousarray(t[:, 1]), np.ascontiguousarray(t[:, 2]))
        return planes, int(math.log2(rgb.shape[0]))
    planes = tuple(np.ascontiguousarray(rgb[..., k]).reshape(-1) for k in range(3))
    return planes, rgb.shape[0]


# ---------------------------------------------------------------- lighting

def vert_light(vn, dirs, ints, amb):
    """vert.vertL for directional lights 1.. (light 0 is shaded per pixel)."""
    vn = vn.astype(np.float32)
    light = np.zeros_like(vn)
    for d, i in zip(dirs[1:], ints[1:]):
        d = np.asarray(d, np.float32)
        dp = (vn[:, 0] * d[0] + vn[:, 1] * d[1]) + vn[:, 2] * d[2]
        light += (np.maximum(np.float32(0), dp + np.float32(0.5)) * np.float32(0.66))[:, None] * np.asarray(i, np.float32)
    return np.maximum(light, np.float32(amb)).astype(np.float32)


SUN = (1.7 * math.pi, 0.52)
LIGHT_DIRS = [view_vec(*SUN), view_vec(SUN[0], SUN[1] + math.pi), view_vec(0, math.pi / 2)]
LIGHT_INTS = [(1.6, 1.4, 1.2), (0.5, 0.5, 0.5), (0.1, 0.2, 0.6)]


def _group(xyz, vn, uv, rgb, flags, amb, alpha_index=0, mip_bias=0.0, cast=True):
    planes, ts = texture_planes(rgb, bool(flags & MIP))
    li = vert_light(vn, LIGHT_DIRS, LIGHT_INTS, amb)
    return Group(np.ascontiguousarray(xyz, np.float32), np.ascontiguousarray(uv, np.float32),
                 np.ascontiguousarray(vn, np.float32), li, planes, ts, flags, alpha_index, mip_bias, cast)


def _finish(groups, alphas, shadows, amb=0.2):
    return Scene(groups, alphas, np.asarray(LIGHT_INTS[0], np.float32),
                 LIGHT_DIRS[0].astype(np.float32), amb, shadows)


# ---------------------------------------------------------------- named scenes

def scene_c1(seed=1, tex=512, terrain_n=64, spheres=200, shadow_dim=1024, flags_extra=0):
    """640x480 plain-view scene: 64x64 terrain (8,192 tris, heights N(0,1)*2)
    + 200 icospheres (16,000 tris); one 512^2 noise texture with mips; one
    1024^2 shadow map."""
    rng = np.random.default_rng(seed)
    xyz, vn, uv = terrain(rng, terrain_n, 1.0, (-terrain_n / 2, 0.0, -terrain_n / 2), 2.0)
    sx, sn, su = icospheres(rng, spheres, 0.2, 1.0, -20, 20)
    rgb, _ = noise_texture(rng, tex)
    f = MIP | SHADOW | flags_extra
    groups = [_group(xyz, vn, uv, rgb, f, 0.2), _group(sx, sn, su, rgb, f | CULL, 0.2)]
    shadows = [ShadowCam.facing(shadow_dim, shadow_dim / 2 / 45.0, (0, 0, 0), SUN)]
    return _finish(groups, [], shadows)


def scene_c3(seed=1):
    """The 24,192-triangle scene of scene_c1 with two cascades (2048^2 and
    1024^2) for the batched multi-view workload."""
    sc = scene_c1(seed=seed)
    sc.shadows = [ShadowCam.facing(2048, 2048 / 2 / 45.0, (0, 0, 0), SUN),
                  ShadowCam.facing(1024, 1024 / 2 / 15.0, (0, 0, 0), SUN)]
    return sc


def scene_c2(seed=2, terrain_n=512, spheres=6000, nquads=20000, tex=2048, alpha_tex=1024, cascades=(2048, 2048)):
    """1080p stress scene: 512x512 terrain (524,288 tris) + 6,000 icospheres
    (480,000) + 20,000 alpha quads (40,000) = 1,044,288 triangles over 5
    materials: 4 trilinear 2048^2 textures, quads on a 1024^2 texture whose
    alpha is thresholded noise; two 2048^2 shadow cascades."""
    rng = np.random.default_rng(seed)
    cell = 128.0 / terrain_n
    xyz, vn, uv = terrain(rng, terrain_n, cell, (-64.0, 0.0, -64.0), 2.0 * cell)
    sx, sn, su = icospheres(rng, spheres, 0.2, 1.0, -20, 20)
    qx, qn, qu = quads(rng, nquads, -20, 20, 0.3, 1.0)
    texs = [noise_texture(rng, tex)[0] for _ in range(4)]
    qrgb, qmask = noise_texture(rng, alpha_tex, alpha_p=0.6)
    half_t = (terrain_n * terrain_n) // 2 * 2 * 3          # vertices in the first half of the cells
    half_s = (spheres // 2) * 80 * 3
    f = MIP | SHADOW
    groups = [
        _group(xyz[:half_t], vn[:half_t], uv[:half_t], texs[0], f, 0.2),
        _group(xyz[half_t:], vn[half_t:], uv[half_t:], texs[1], f, 0.2),
        _group(sx[:half_s], sn[:half_s], su[:half_s], texs[2], f | CULL, 0.2),
        _group(sx[half_s:], sn[half_s:], su[half_s:], texs[3], f | CULL, 0.2),
        _group(qx, qn, qu, qrgb, ALPHA | SHADOW, 0.2, alpha_index=0),
    ]
    shadows = [ShadowCam.facing(cascades[0], cascades[0] / 2 / 24.0, (0, 0, 0), SUN),
               ShadowCam.facing(cascades[1], cascades[1] / 2 / 72.0, (0, 0, 0), SUN)]
    return _finish(groups, [(qmask.reshape(-1), alpha_tex)], shadows)


def scene_small(seed=3, terrain_n=16, spheres=24, nquads=40, tex=64, alpha_tex=64, shadow_dim=256,
                flags=MIP | SHADOW, with_alpha=True):
    """Small mixed scene for parity tests (seconds on the oracle)."""
    rng = np.random.default_rng(seed)
    xyz, vn, uv = terrain(rng, terrain_n, 2.0, (-terrain_n, 0.0, -terrain_n), 1.0)
    sx, sn, su = icospheres(rng, spheres, 0.5, 2.5, -12, 12)
    rgb, _ = noise_texture(rng, tex)
    groups = [_group(xyz, vn, uv, rgb, flags, 0.2), _group(sx, sn, su, rgb, flags | CULL, 0.2)]
    alphas = []
    if with_alpha:
        qx, qn, qu = quads(rng, nquads, -10, 10, 1.0, 4.0)
        qrgb, qmask = noise_texture(rng, alpha_tex, alpha_p=0.6)
        groups.append(_group(qx, qn, qu, qrgb, (flags & ~MIP) | ALPHA, 0.2, alpha_index=0))
        alphas.append((qmask.reshape(-1), alpha_tex))
    shadows = [ShadowCam.facing(shadow_dim, shadow_dim / 2 / 30.0, (0, 0, 0), SUN),
               ShadowCam.facing(shadow_dim // 2, shadow_dim / 4 / 60.0, (0, 0, 0), SUN)]
    return _finish(groups, alphas, shadows)


def scene_multi(seed=9, terrain_n=24, cell=2.0, tex=64, spheres=12, shadow_dim=256):
    """A terrain in the 4-way blend material (av_draw_multi.c, as
    PyOpenCL27C/3RandTerrain2.py uses it): heights from 0 to about 25 so the
    sand (y < 5), rock (y > 15) and snow (y > 16 + ripple) weights and the
    normal-dependent terms all occur.  Groups 1-3 are single quads whose
    textures the blend samples (the demo's Rock, Snow and Sand planes);
    group 4 is icospheres in the trilinear + shadow material."""
    rng = np.random.default_rng(seed)
    n = terrain_n
    i = np.arange(n + 1)
    hx, hz = np.meshgrid(i, i, indexing="ij")
    h = 12.5 + 9.0 * np.sin(hx * 0.45 + rng.uniform(0, 6)) * np.cos(hz * 0.35 + rng.uniform(0, 6))
    h += rng.standard_normal(h.shape) * 1.5
    xyz, vn, uv = terrain_from_heights(h, cell, (-n * cell / 2, 0.0, -n * cell / 2), 1.0)
    grass, _ = noise_texture(rng, tex)
    groups = [_group(xyz, vn, uv, grass, MULTI | CULL, 0.2)]
    for k in range(3):
        qx, qn, qu = quads(rng, 1, -4, 4, 1.0, 2.0, ground=3.0 * k)
        rgb, _ = noise_texture(rng, tex)
        groups.append(_group(qx, qn, qu, rgb, 0, 0.2))
    sx, sn, su = icospheres(rng, spheres, 0.5, 2.0, -n * cell / 3, n * cell / 3)
    sx[:, 1] += 14.0
    srgb, _ = noise_texture(rng, tex)
    groups.append(_group(sx, sn, su, srgb, MIP | SHADOW | CULL, 0.2))
    shadows = [ShadowCam.facing(shadow_dim, shadow_dim / 2 / 30.0, (0, 10, 0), SUN),
               ShadowCam.facing(shadow_dim // 2, shadow_dim / 4 / 60.0, (0, 10, 0), SUN)]
    return _finish(groups, [], shadows)


def noise_rgb_fast(rng, n):
    """n x n RGB uniform noise preprocessed as c*c/8 (uint16), computed in
    integers (exact: c*c <= 65025), for the large textures of the stress
    scene."""
    c = rng.integers(0, 256, (n, n, 3), dtype=np.uint16).astype(np.uint32)
    return ((c * c) >> 3).astype(np.uint16)


def scene_c5(seed=5, terrain_n=2048, spheres=20000, tex=4096, terrain_groups=12, sphere_groups=4,
             alpha_terrain=(2, 5, 8), alpha_spheres=(0, 2), cascades=(4096, 4096), extent=128.0):
    """3840x2160 stress scene: a 2048x2048 terrain (8,388,608 tris) in 12
    row bands plus 20,000 icospheres (1,600,000) in 4 groups = 9,988,608
    triangles over 16 materials, each with its own 4096^2 trilinear noise
    texture; 3 terrain bands and 2 sphere groups (29% of the triangles) are
    alpha-tested against one 4096^2 thresholded-noise mask; two 4096^2
    cascades (64 and 256 units across)."""
    rng = np.random.default_rng(seed)
    cell = 2 * extent / terrain_n
    xyz, vn, uv = terrain(rng, terrain_n, cell, (-extent, 0.0, -extent), 2.0 * cell)
    sx, sn, su = icospheres(rng, spheres, 0.2, 1.0, -extent * 0.3, extent * 0.3)
    amask = (rng.random((tex, tex)) < 0.6).astype(np.uint8)        # alpha 255 (kept) with p = 0.6
    groups = []
    f = MIP | SHADOW
    nt = len(xyz) // 3
    for k in range(terrain_groups):
        a, b = 3 * (nt * k // terrain_groups), 3 * (nt * (k + 1) // terrain_groups)
        fl = f | (ALPHA if k in alpha_terrain else 0)
        groups.append(_group(xyz[a:b], vn[a:b], uv[a:b], noise_rgb_fast(rng, tex), fl, 0.2))
    ns = len(sx) // 3
    for k in range(sphere_groups):
        a, b = 3 * (ns * k // sphere_groups), 3 * (ns * (k + 1) // sphere_groups)
        fl = f | CULL | (ALPHA if k in alpha_spheres else 0)
        groups.append(_group(sx[a:b], sn[a:b], su[a:b], noise_rgb_fast(rng, tex), fl, 0.2))
    shadows = [ShadowCam.facing(cascades[0], cascades[0] / 2 / 32.0, (0, 0, 0), SUN),
               ShadowCam.facing(cascades[1], cascades[1] / 2 / 128.0, (0, 0, 0), SUN)]
    return _finish(groups, [(amask.reshape(-1), tex)], shadows)


SERVING_SEEDS = tuple(range(10, 18))


def scene_served(seed, tmin=50_000, tmax=1_000_000, tex=1024, alpha_tex=512, cascades=(2048, 1024)):
    """One of the resident scenes of the serving workload: a triangle budget T
    drawn log-uniform in [tmin, tmax] from the seed, split about half terrain,
    45% icospheres, 5% alpha-tested quads, over 4 materials (two trilinear
    terrain/sphere textures, one sphere material without mip, the alpha quads);
    two shadow cascades of the same sun."""
    rng = np.random.default_rng(seed)
    T = float(np.exp(rng.uniform(math.log(tmin), math.log(tmax))))
    n = max(8, int(round(math.sqrt(T * 0.5 / 2))))
    spheres = max(2, int(T * 0.45 / 80))
    nquads = max(2, int(T * 0.05 / 2))
    extent = 16.0 + 48.0 * math.sqrt(T / tmax)
    cell = 2 * extent / n
    xyz, vn, uv = terrain(rng, n, cell, (-extent, 0.0, -extent), 2.0 * cell)
    sx, sn, su = icospheres(rng, spheres, 0.2, 1.0, -extent * 0.6, extent * 0.6)
    qx, qn, qu = quads(rng, nquads, -extent * 0.6, extent * 0.6, 0.3, 1.0)
    texs = [noise_texture(rng, tex)[0] for _ in range(3)]
    qrgb, qmask = noise_texture(rng, alpha_tex, alpha_p=0.6)
    half_s = (spheres // 2) * 80 * 3
    f = MIP | SHADOW
    groups = [
        _group(xyz, vn, uv, texs[0], f, 0.2),
        _group(sx[:half_s], sn[:half_s], su[:half_s], texs[1], f | CULL, 0.2),
        _group(sx[half_s:], sn[half_s:], su[half_s:], texs[2], SHADOW | CULL, 0.2),
        _group(qx, qn, qu, qrgb, ALPHA | SHADOW, 0.2, alpha_index=0),
    ]
    shadows = [ShadowCam.facing(cascades[0], cascades[0] / 2 / (extent * 0.75), (0, 0, 0), SUN),
               ShadowCam.facing(cascades[1], cascades[1] / 2 / (extent * 1.5), (0, 0, 0), SUN)]
    return _finish(groups, [(qmask.reshape(-1), alpha_tex)], shadows)


def scene_normal(seed=6, terrain_n=16, spheres=20, nquads=30, tex=64, shadow_dim=256):
    """The normal-mapped materials on one raster (av_draw_normmap.c,
    _alpha.c, _mip.c): terrain with a normal map (roughness 0.5), metal
    icospheres (roughness 0.3) and trilinear icospheres with a normal-map
    chain (mipBias 0.4), alpha-tested quads with a normal map; two cascades
    (the normal-mapped materials sample the first)."""
    rng = np.random.default_rng(seed)
    xyz, vn, uv = terrain(rng, terrain_n, 2.0, (-terrain_n, 0.0, -terrain_n), 1.0)
    sx, sn, su = icospheres(rng, spheres, 0.5, 2.5, -12, 12)
    qx, qn, qu = quads(rng, nquads, -10, 10, 1.0, 4.0)
    rgb, _ = noise_texture(rng, tex)
    qrgb, qmask = noise_texture(rng, tex, alpha_p=0.6)
    half = (spheres // 2) * 80 * 3
    groups = [_group(xyz, vn, uv, rgb, NORMAL | SHADOW, 0.2),
              _group(sx[:half], sn[:half], su[:half], rgb, NORMAL | SHADOW | CULL, 0.2),
              _group(sx[half:], sn[half:], su[half:], rgb, NORMAL | MIP | SHADOW | CULL, 0.2, mip_bias=0.4),
              _group(qx, qn, qu, qrgb, NORMAL | ALPHA | SHADOW, 0.2, alpha_index=0)]
    for g, rough, metal in zip(groups, (0.5, 0.3, 0.5, 0.7), (False, True, False, False)):
        g.nm = normal_map(rng, tex, bool(g.flags & MIP))
        g.roughness, g.metal = rough, metal
    shadows = [ShadowCam.facing(shadow_dim, shadow_dim / 2 / 30.0, (0, 0, 0), SUN),
               ShadowCam.facing(shadow_dim // 2, shadow_dim / 4 / 60.0, (0, 0, 0), SUN)]
    return _finish(groups, [(qmask.reshape(-1), tex)], shadows)


def default_view(w, h, pos=(0.0, 5.0, -25.0), target=(0.0, 0.0, 0.0), fov=70.0):
    return View.perspective(w, h, pos, target, fov)


def reference_kernel_variant(scene):
    """The same geometry with only what the reference's existing draw kernels
    support (PyOpenCL27C/Shaders/drawtexcolsmp.c, drawtexcolsmpalpha.c):
    mip groups sample their full-resolution level bilinearly and no shadow
    lookup is made.  Used to run the reference's own kernels on a scene."""
    groups = []
    for g in scene.groups:
        r, gg, b = g.tex
        ts = g.tex_size
        if g.flags & MIP:
            side = 1 << g.tex_size
            base = (side * side - 1) // 3            # texels of the smaller levels
            r, gg, b = (np.ascontiguousarray(x[base:base + side * side]) for x in (r, gg, b))
            ts = side
        groups.append(Group(g.xyz, g.uv, g.vn, g.li, (r, gg, b), ts, g.flags & ~(MIP | SHADOW),
                            g.alpha_index, g.mip_bias, g.cast))
    return Scene(groups, scene.alphas, scene.lint, scene.ldir, scene.amb, scene.shadows, scene.bias)
