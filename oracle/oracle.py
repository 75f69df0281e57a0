"""ctypes bindings for the CPU oracle (liboracle_axr.so) and for the
reference kernels compiled for the CPU (oracle/_ref/libaxr_ref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py.  The product package never
imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle_axr.so")
REF_SO = os.path.join(HERE, "_ref", "libaxr_ref.so")

CFLAGS = ["-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math", "-fopenmp"]


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "axr_oracle.c")
    if force or not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < max(
            os.path.getmtime(src), os.path.getmtime(os.path.join(HERE, "axr_oracle.h"))):
        subprocess.run(["gcc", *CFLAGS, "-o", ORACLE_SO, src, "-lm"], check=True)
    return ORACLE_SO


class OrcGroup(C.Structure):
    _fields_ = [("ntris", C.c_int), ("xyz", C.c_void_p), ("vn", C.c_void_p), ("uv", C.c_void_p),
                ("li", C.c_void_p), ("tr", C.c_void_p), ("tg", C.c_void_p), ("tb", C.c_void_p),
                ("tex_size", C.c_int), ("flags", C.c_int), ("alpha_index", C.c_int), ("mip_bias", C.c_float),
                ("nm", C.c_void_p), ("roughness", C.c_float), ("is_metal", C.c_int)]


class OrcAlpha(C.Structure):
    _fields_ = [("mask", C.c_void_p), ("len", C.c_int)]


class OrcShadow(C.Structure):
    _fields_ = [("map", C.c_void_p), ("dim", C.c_int), ("scale", C.c_float),
                ("pos", C.c_float * 3), ("vv", C.c_float * 9)]


class OrcFrame(C.Structure):
    _fields_ = [("w", C.c_int), ("h", C.c_int), ("pos", C.c_float * 3), ("vv", C.c_float * 9),
                ("sscale", C.c_float), ("cax", C.c_float), ("cay", C.c_float),
                ("lint", C.c_float * 3), ("ldir", C.c_float * 3), ("amb", C.c_float),
                ("ro", C.c_void_p), ("go", C.c_void_p), ("bo", C.c_void_p), ("db", C.c_void_p),
                ("tri_id", C.c_void_p), ("cov", C.c_void_p)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build_oracle()                  # rebuilds only when the source is newer
        L = C.CDLL(ORACLE_SO)
        L.orc_draw_all.restype = C.c_int
        L.orc_draw_all.argtypes = [C.POINTER(OrcFrame), C.POINTER(OrcGroup), C.c_int, C.c_void_p,
                                   C.POINTER(OrcAlpha), C.c_int, C.POINTER(OrcShadow), C.c_int, C.c_int]
        L.orc_shadow_map.restype = C.c_int
        L.orc_shadow_map.argtypes = [C.POINTER(OrcShadow), C.POINTER(OrcGroup), C.c_int, C.c_void_p,
                                     C.POINTER(OrcAlpha), C.c_int, C.c_float, C.c_int]
        L.orc_clear_depth.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
        L.orc_gamma.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_float]
        L.orc_setup_persp.argtypes = [C.POINTER(OrcGroup), C.POINTER(OrcFrame), C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_coarse_counts.restype = C.c_long
        L.orc_coarse_counts.argtypes = [C.POINTER(OrcGroup), C.POINTER(OrcFrame), C.c_void_p]
        L.orc_log2f.restype = C.c_float
        L.orc_log2f.argtypes = [C.c_float]
        L.orc_ssao.argtypes = [C.c_void_p] * 4 + [C.c_int, C.c_int, C.c_float, C.c_void_p]
        L.orc_dof.argtypes = [C.c_void_p] * 4 + [C.c_int, C.c_int, C.c_float] + [C.c_void_p] * 3
        L.orc_bloom.argtypes = [C.c_void_p] * 3 + [C.c_int, C.c_int]
        L.orc_transform.argtypes = [C.c_void_p] * 5 + [C.c_int, C.c_int]
        L.orc_translate.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        L.orc_vert_light.argtypes = ([C.c_void_p] * 3 + [C.c_int] + [C.c_void_p] * 2 + [C.c_int]
                                     + [C.c_void_p] * 2 + [C.c_int] + [C.c_void_p] * 3 + [C.c_int, C.c_float])
        _lib = L
    return _lib


def _ptr(a):
    """Address of an array's data.  The caller keeps the array referenced
    until the C call returns (a temporary is freed as soon as this returns)."""
    return a.ctypes.data if a is not None else None


def _v3(a, n=None):
    """float32 C-contiguous (k, 3) array (k = 0 for None)."""
    if a is None:
        return np.zeros((0, 3), np.float32)
    return np.ascontiguousarray(np.asarray(a, np.float32).reshape(-1, 3))


def _m3(a):
    return np.ascontiguousarray(np.asarray(a, np.float32).reshape(3, 3))


def ssao(fr, sscale, rnd):
    """Post/ssao.c on a Frame's colour planes, in place (depth read only)."""
    t = np.ascontiguousarray(np.asarray(rnd, np.float32).reshape(-1)[:32])
    lib().orc_ssao(_ptr(fr.ro), _ptr(fr.go), _ptr(fr.bo), _ptr(fr.db), fr.w, fr.h, C.c_float(sscale), _ptr(t))


def dof(fr, focus):
    """Post/dof.c on a Frame: the gathered region replaces the colour planes;
    pixels outside the (w/16*16) x (h/16*16) region keep their colour."""
    r2, g2, b2 = fr.ro.copy(), fr.go.copy(), fr.bo.copy()
    lib().orc_dof(_ptr(fr.ro), _ptr(fr.go), _ptr(fr.bo), _ptr(fr.db), fr.w, fr.h, C.c_float(focus),
                  _ptr(r2), _ptr(g2), _ptr(b2))
    fr.ro, fr.go, fr.bo = r2, g2, b2


def bloom(fr):
    """Post/blur.c + Post/blur2.c (CLDraw.blur) on a Frame's colour planes, in place."""
    lib().orc_bloom(_ptr(fr.ro), _ptr(fr.go), _ptr(fr.bo), fr.w, fr.h)


def transform(xyz, vn, old_rm, rot_mat, origin, start=0, end=None):
    """vert.transform on packed (V, 3) float32 arrays, in place (CLDraw.rotate)."""
    end = xyz.shape[0] if end is None else end
    o = np.asarray(origin, np.float32).reshape(3)
    old, rot = _m3(old_rm), _m3(rot_mat)            # held until the call returns
    lib().orc_transform(_ptr(xyz), _ptr(vn), _ptr(old), _ptr(rot), _ptr(o), start, end)


def translate(xyz, coords, start=0, end=None):
    """vert.Ttranslate on a packed (V, 3) float32 array, in place."""
    end = xyz.shape[0] if end is None else end
    c = np.asarray(coords, np.float32).reshape(3)
    lib().orc_translate(_ptr(xyz), _ptr(c), start, end)


def vert_light(xyz, vn, dir_int, dir_dir, amb, point_int=None, point_pos=None,
               spot_int=None, spot_dir=None, spot_pos=None):
    """vert.vertL: the per-vertex light I of (V, 3) positions and normals."""
    di, dd, pi, pp, si, sd, sp = (_v3(a) for a in (dir_int, dir_dir, point_int, point_pos, spot_int, spot_dir,
                                                   spot_pos))
    x, n = np.ascontiguousarray(xyz, np.float32), np.ascontiguousarray(vn, np.float32)
    li = np.empty_like(n)
    lib().orc_vert_light(_ptr(x), _ptr(n), _ptr(li), li.shape[0], _ptr(di), _ptr(dd), di.shape[0], _ptr(pi), _ptr(pp), pi.shape[0],
                         _ptr(si), _ptr(sd), _ptr(sp), si.shape[0], C.c_float(amb))
    return li


class Frame:
    """Host framebuffers for one view (reference layout: u16 planes, f32 depth)."""

    def __init__(self, w, h):
        self.w, self.h = w, h
        self.ro = np.ones((h, w), np.uint16)
        self.go = np.ones((h, w), np.uint16)
        self.bo = np.ones((h, w), np.uint16)
        self.db = np.full((h, w), 65535.0, np.float32)
        self.tri_id = np.full((h, w), -1, np.int32)
        self.cov = np.zeros((h, w), np.uint8)


def _groups(scene):
    arr = (OrcGroup * len(scene.groups))()
    keep = []
    for k, g in enumerate(scene.groups):
        r, gg, b = g.tex
        nm = getattr(g, "nm", None)
        keep += [g.xyz, g.vn, g.uv, g.li, r, gg, b, nm]
        arr[k] = OrcGroup(g.ntris, _ptr(g.xyz), _ptr(g.vn), _ptr(g.uv), _ptr(g.li), _ptr(r), _ptr(gg), _ptr(b),
                          g.tex_size, g.flags, g.alpha_index, g.mip_bias, _ptr(nm) if nm is not None else None,
                          getattr(g, "roughness", 0.0), int(getattr(g, "metal", False)))
    return arr, keep


def _alphas(scene):
    n = max(1, len(scene.alphas))
    arr = (OrcAlpha * n)()
    keep = []
    for k, (m, ln) in enumerate(scene.alphas):
        m = np.ascontiguousarray(m, np.uint8)
        keep.append(m)
        arr[k] = OrcAlpha(_ptr(m), ln)
    return arr, keep


def _shadow_struct(sc, m):
    s = OrcShadow()
    s.map = _ptr(m)
    s.dim = sc.dim
    s.scale = sc.scale
    s.pos[:] = [float(x) for x in sc.pos]
    s.vv[:] = [float(x) for x in np.asarray(sc.vv, np.float32).reshape(-1)]
    return s


def new_shadow_map(dim):
    return np.full((dim, dim), 65535.0, np.float32)


def shadow_map(scene, k, smap, cast=None, nthreads=1):
    """CLDraw.shadowMap(k, ...) on the oracle; smap is updated in place."""
    L = lib()
    sc = scene.shadows[k]
    s = _shadow_struct(sc, smap)
    g, keep = _groups(scene)
    a, keep2 = _alphas(scene)
    if cast is None:
        cast = [gr.cast for gr in scene.groups]
    cast = np.asarray(cast, np.uint8)
    rc = L.orc_shadow_map(C.byref(s), g, len(scene.groups), _ptr(cast), a, len(scene.alphas),
                          C.c_float(scene.bias), nthreads)
    if rc != 0:
        raise RuntimeError(f"orc_shadow_map failed: {rc}")
    return smap


def _frame_struct(fr, view, scene):
    f = OrcFrame()
    f.w, f.h = view.w, view.h
    f.pos[:] = [float(x) for x in view.pos]
    f.vv[:] = [float(x) for x in np.asarray(view.vv, np.float32).reshape(-1)]
    f.sscale, f.cax, f.cay = view.sscale, view.cax, view.cay
    f.lint[:] = [float(x) for x in scene.lint]
    f.ldir[:] = [float(x) for x in scene.ldir]
    f.amb = scene.amb
    f.ro, f.go, f.bo, f.db = _ptr(fr.ro), _ptr(fr.go), _ptr(fr.bo), _ptr(fr.db)
    f.tri_id, f.cov = _ptr(fr.tri_id), _ptr(fr.cov)
    return f


def draw_all(scene, view, fr, smaps=(), mask=None, nthreads=1):
    """CLDraw.drawAll on the oracle: updates `fr` (a Frame) in place."""
    L = lib()
    f = _frame_struct(fr, view, scene)
    g, keep = _groups(scene)
    a, keep2 = _alphas(scene)
    n_sh = len(smaps)
    sh = (OrcShadow * max(1, n_sh))()
    for k in range(n_sh):
        sh[k] = _shadow_struct(scene.shadows[k], smaps[k])
    m = None if mask is None else np.asarray(mask, np.uint8)
    rc = L.orc_draw_all(C.byref(f), g, len(scene.groups), _ptr(m), a, len(scene.alphas), sh, n_sh, nthreads)
    if rc != 0:
        raise RuntimeError(f"orc_draw_all failed: {rc}")
    return fr


def clear_depth(db, lenP=4):
    h, w = db.shape
    lib().orc_clear_depth(_ptr(db), w, h, lenP)


def gamma(fr, exposure=1.0):
    lib().orc_gamma(_ptr(fr.ro), _ptr(fr.go), _ptr(fr.bo), fr.w, fr.h, C.c_float(exposure))


def render(scene, view, nthreads=1, with_shadows=True):
    """Full frame on the oracle: shadow maps, clear, drawAll.  Returns
    (Frame, shadow maps)."""
    smaps = []
    if with_shadows:
        for k, sc in enumerate(scene.shadows):
            m = new_shadow_map(sc.dim)
            shadow_map(scene, k, m, nthreads=nthreads)
            smaps.append(m)
    fr = Frame(view.w, view.h)
    clear_depth(fr.db)
    draw_all(scene, view, fr, smaps, nthreads=nthreads)
    return fr, smaps


def setup_persp(scene, gi, view):
    L = lib()
    g, keep = _groups(scene)
    fr = Frame(view.w, view.h)
    f = _frame_struct(fr, view, scene)
    n = scene.groups[gi].ntris
    cls = np.zeros(n, np.uint8)
    sp = np.zeros((n * 3, 2), np.float32)
    zz = np.zeros(n * 3, np.float32)
    L.orc_setup_persp(C.byref(g[gi]), C.byref(f), _ptr(cls), _ptr(sp), _ptr(zz))
    return cls, sp, zz


def coarse_counts(scene, gi, view):
    L = lib()
    g, keep = _groups(scene)
    fr = Frame(view.w, view.h)
    f = _frame_struct(fr, view, scene)
    counts = np.zeros((view.h // 16) * (view.w // 16), np.int32)
    total = L.orc_coarse_counts(C.byref(g[gi]), C.byref(f), _ptr(counts))
    return total, counts


# ---------------------------------------------------------------- reference kernels on the CPU

_ref = None


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        R = C.CDLL(REF_SO)
        R.ref_create.restype = C.c_void_p
        R.ref_create.argtypes = [C.c_int, C.c_int]
        R.ref_destroy.argtypes = [C.c_void_p]
        R.ref_add_group.restype = C.c_int
        R.ref_add_group.argtypes = [C.c_void_p] + [C.c_void_p] * 4 + [C.c_int] + [C.c_void_p] * 3 + [C.c_long, C.c_int]
        R.ref_add_alpha.restype = C.c_int
        R.ref_add_alpha.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        R.ref_set_view.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_float]
        R.ref_set_light.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        R.ref_clear_zbuffer.argtypes = [C.c_void_p]
        R.ref_set_depth.argtypes = [C.c_void_p, C.c_void_p]
        R.ref_draw_all.restype = C.c_int
        R.ref_draw_all.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        R.ref_get_frame.argtypes = [C.c_void_p] + [C.c_void_p] * 4
        R.ref_set_frame.argtypes = [C.c_void_p] + [C.c_void_p] * 3
        R.ref_add_shadow_map.restype = C.c_int
        R.ref_add_shadow_map.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float]
        R.ref_place_shadow_map.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        R.ref_clear_shadow_map.argtypes = [C.c_void_p, C.c_int]
        R.ref_shadow_map.restype = C.c_int
        R.ref_shadow_map.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float, C.c_int]
        R.ref_get_shadow_map.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        R.ref_gamma.argtypes = [C.c_void_p, C.c_float]
        R.ref_overflow.restype = C.c_int
        R.ref_overflow.argtypes = [C.c_void_p]
        R.ref_transform.restype = C.c_int
        R.ref_transform.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 3 + [C.c_int, C.c_int]
        R.ref_translate.restype = C.c_int
        R.ref_translate.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int]
        R.ref_vert_light.restype = C.c_int
        R.ref_vert_light.argtypes = ([C.c_void_p, C.c_void_p, C.c_int] + [C.c_void_p] * 2 + [C.c_int]
                                     + [C.c_void_p] * 2 + [C.c_int] + [C.c_void_p] * 3 + [C.c_int, C.c_float])
        R.ref_ssao.argtypes = [C.c_void_p, C.c_void_p]
        R.ref_bloom.argtypes = [C.c_void_p]
        R.ref_dof.argtypes = [C.c_void_p, C.c_float]
        R.ref_set_normal.restype = C.c_int
        R.ref_set_normal.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_long, C.c_float, C.c_int, C.c_float]
        R.ref_set_normal_shadow.argtypes = [C.c_void_p, C.c_int]
        R.ref_set_mip_kernels.restype = C.c_int
        R.ref_set_mip_kernels.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int]
        R.ref_get_geometry.restype = C.c_int
        R.ref_get_geometry.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 3
        _ref = R
    return _ref


class RefDraw:
    """The reference's CLDraw, run through its own kernels on the CPU."""

    def __init__(self, scene, view):
        self.R = ref_lib()
        self.scene, self.view = scene, view
        self.h = self.R.ref_create(view.w, view.h)
        self._keep = []
        for g in scene.groups:
            r, gg, b = g.tex
            self.R.ref_add_group(self.h, _ptr(g.xyz), _ptr(g.uv), _ptr(g.vn), _ptr(g.li), g.ntris,
                                 _ptr(r), _ptr(gg), _ptr(b), r.size, g.tex_size)
        for m, ln in scene.alphas:
            m = np.ascontiguousarray(m, np.uint8)
            self.R.ref_add_alpha(self.h, _ptr(m), ln)
        pos = np.asarray(view.pos, np.float32)
        vv = np.ascontiguousarray(view.vv, np.float32)
        self.R.ref_set_view(self.h, _ptr(pos), _ptr(vv), view.sscale, view.cax, view.cay)
        self._light = (np.asarray(scene.lint, np.float32), np.asarray(scene.ldir, np.float32))
        self.R.ref_set_light(self.h, _ptr(self._light[0]), _ptr(self._light[1]))
        self.flags = np.array([g.flags for g in scene.groups], np.int32)
        self.aidx = np.array([g.alpha_index for g in scene.groups], np.int32)
        # the normal-mapped materials (flags bit 5): their maps, and the
        # first cascade as the one they sample
        for k, g in enumerate(scene.groups):
            if g.flags & 32:
                nm = np.ascontiguousarray(g.nm, np.uint8)
                self._keep.append(nm)
                if self.R.ref_set_normal(self.h, k, _ptr(nm), nm.size // 4, g.roughness, int(g.metal),
                                         g.mip_bias) != 0:
                    raise RuntimeError(f"ref_set_normal: group {k}")
        self.R.ref_set_normal_shadow(self.h, 0 if scene.shadows else -1)

    def __del__(self):
        try:
            self.R.ref_destroy(self.h)
        except Exception:
            pass

    def set_mip_kernels(self, on=True):
        """Draw the mip groups with the reference's normal-mapped mip material
        (Shaders_src/av_draw_normmap_mip.c as its AVSL generator expands it),
        each group with its mipBias."""
        bias = np.array([g.mip_bias for g in self.scene.groups], np.float32)
        if self.R.ref_set_mip_kernels(self.h, 1 if on else 0, _ptr(bias), len(bias)) != 0:
            raise RuntimeError("ref_set_mip_kernels")

    def clear_zbuffer(self):
        self.R.ref_clear_zbuffer(self.h)

    def draw_all(self, mask=None, nthreads=1):
        m = None if mask is None else np.asarray(mask, np.uint8)
        rc = self.R.ref_draw_all(self.h, _ptr(self.flags), _ptr(self.aidx), _ptr(m), len(self.flags), nthreads)
        return rc

    def get_frame(self):
        w, h = self.view.w, self.view.h
        r = np.empty((h, w), np.uint16); g = np.empty((h, w), np.uint16); b = np.empty((h, w), np.uint16)
        db = np.empty((h, w), np.float32)
        self.R.ref_get_frame(self.h, _ptr(r), _ptr(g), _ptr(b), _ptr(db))
        return r, g, b, db

    def shadow_map(self, k, cast=None, nthreads=1, clear=True, read=True):
        """Renders the casters into shadow map k; clear=False draws over the
        map's current contents, read=False skips the copy out."""
        sc = self.scene.shadows[k]
        if clear:
            self.R.ref_add_shadow_map(self.h, k, sc.dim, sc.scale)
            p, vv = np.asarray(sc.pos, np.float32), np.ascontiguousarray(sc.vv, np.float32)
            self.R.ref_place_shadow_map(self.h, k, _ptr(p), _ptr(vv))
            self.R.ref_clear_shadow_map(self.h, k)
        if cast is None:
            cast = [g.cast for g in self.scene.groups]
        cast = np.asarray(cast, np.uint8)
        rc = self.R.ref_shadow_map(self.h, k, _ptr(cast), _ptr(self.flags), _ptr(self.aidx), len(self.flags),
                                   self.scene.bias, nthreads)
        if not read:
            return rc, None
        out = np.empty((sc.dim, sc.dim), np.float32)
        self.R.ref_get_shadow_map(self.h, k, _ptr(out))
        return rc, out

    def gamma(self, ex=1.0):
        self.R.ref_gamma(self.h, ex)

    # vertex stage (Pipe/vert.c through CLDraw.rotate / translate / vertLight)
    def rotate(self, old_rm, rot_mat, origin, start, end, tn):
        o = np.asarray(origin, np.float32).reshape(3)
        old, rot = _m3(old_rm), _m3(rot_mat)
        return self.R.ref_transform(self.h, tn, _ptr(old), _ptr(rot), _ptr(o), start, end)

    def translate(self, coords, start, end, tn):
        c = np.asarray(coords, np.float32).reshape(3)
        return self.R.ref_translate(self.h, tn, _ptr(c), start, end)

    def vert_light(self, mask, dir_int, dir_dir, amb, point_int=None, point_pos=None,
                   spot_int=None, spot_dir=None, spot_pos=None):
        di, dd, pi, pp, si, sd, sp = (_v3(a) for a in (dir_int, dir_dir, point_int, point_pos, spot_int,
                                                       spot_dir, spot_pos))
        m = np.asarray(mask, np.uint8)
        return self.R.ref_vert_light(self.h, _ptr(m), len(m), _ptr(di), _ptr(dd), di.shape[0], _ptr(pi), _ptr(pp),
                                     pi.shape[0], _ptr(si), _ptr(sd), _ptr(sp), si.shape[0], C.c_float(amb))

    def geometry(self, tn):
        nv = self.scene.groups[tn].ntris * 3
        xyz = np.empty((nv, 3), np.float32); vn = np.empty((nv, 3), np.float32); li = np.empty((nv, 3), np.float32)
        self.R.ref_get_geometry(self.h, tn, _ptr(xyz), _ptr(vn), _ptr(li))
        return xyz, vn, li

    # post effects (Post/ssao.c, Post/dof.c)
    def ssao(self, rnd):
        t = np.zeros(48, np.float32)
        t[:32] = np.asarray(rnd, np.float32).reshape(-1)[:32]
        self.R.ref_ssao(self.h, _ptr(t))

    def dof(self, focus):
        self.R.ref_dof(self.h, C.c_float(focus))

    def bloom(self):
        self.R.ref_bloom(self.h)

    def set_frame(self, r, g, b, db):
        """Replaces the colour planes and the depth buffer."""
        arrs = [np.ascontiguousarray(a) for a in (r, g, b)]
        d = np.ascontiguousarray(db, np.float32)
        self.R.ref_set_frame(self.h, *[_ptr(a) for a in arrs])
        self.R.ref_set_depth(self.h, _ptr(d))
