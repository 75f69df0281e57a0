"""Batched multi-view rendering: many views of uneven size -- shaded
perspective views (main view, cubemap faces) and depth-only shadow cascades
that those views sample -- rendered by one persistent cooperative launch
replayed from a captured CUDA graph (include/axr.h, axr_batch_*).

Each view's result equals rendering it alone through CLDraw.drawAll /
shadowMap, bit for bit.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._lib import ViewDesc, check, lib
from . import scenes as S

SHADED, DEPTH, SKIP = 0, 1, 2
PERSISTENT, PHASED = 0, 1


def _groups(d, groups):
    if groups is not None:
        d.group_first, d.group_count = int(groups[0]), int(groups[1])
    return d


def shaded(view: S.View, cascades=(), groups=None, clear=None):
    """A shaded view sampling `cascades` (batch view indices, or -1-i for the
    handle's shadow map i), drawing the group range groups = (first, count)
    (None: every group); clear = (r, g, b) fills the colour planes first."""
    d = ViewDesc()
    d.kind, d.w, d.h = SHADED, view.w, view.h
    d.pos[:] = [float(x) for x in view.pos]
    d.vm[:] = [float(x) for x in np.asarray(view.vv, np.float32).reshape(-1)]
    d.scale, d.cax, d.cay = view.sscale, view.cax, view.cay
    d.ncascades = len(cascades)
    for k, c in enumerate(cascades):
        d.cascades[k] = int(c)
    if clear is not None:
        d.clear_color = 1
        d.bg[:] = [int(x) for x in clear]
    return _groups(d, groups)


def skip(w, h):
    """An unused shaded slot of size w x h."""
    d = ViewDesc()
    d.kind, d.w, d.h = SKIP, w, h
    return d


def depth(cam: S.ShadowCam, bias: float, groups=None):
    d = ViewDesc()
    d.kind, d.w, d.h = DEPTH, cam.dim, cam.dim
    d.pos[:] = [float(x) for x in cam.pos]
    d.vm[:] = [float(x) for x in np.asarray(cam.vv, np.float32).reshape(-1)]
    d.scale = cam.scale
    d.bias = float(np.float32(bias))
    return _groups(d, groups)


# camera angles (alpha, beta) of the six cube faces: +x, -x, +y, -y, +z, -z
CUBE_FACES = [(math.pi / 2, 0.0), (-math.pi / 2, 0.0), (0.0, -math.pi / 2 + 1e-4), (0.0, math.pi / 2 - 1e-4),
              (0.0, 0.0), (math.pi, 0.0)]


def cube_faces(pos, side=512):
    """Six 90-degree perspective views around `pos`."""
    return [S.View.perspective(side, side, pos, fov_deg=90.0, angles=a) for a in CUBE_FACES]


class Batch:
    def __init__(self, draw, descs):
        self.draw = draw
        self._L = lib()
        self.descs = list(descs)
        arr = (ViewDesc * len(self.descs))(*self.descs)
        h = C.c_void_p()
        check(self._L.axr_batch_create(draw._h, arr, len(self.descs), C.byref(h)), "axr_batch_create")
        self._h = h

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                self._L.axr_batch_destroy(self._h)
                self._h = None
        except Exception:
            pass

    def set_views(self, descs):
        self.descs = list(descs)
        arr = (ViewDesc * len(self.descs))(*self.descs)
        check(self._L.axr_batch_set_views(self._h, arr, len(self.descs)), "axr_batch_set_views")

    def set_views_array(self, arr):
        """set_views from a ctypes ViewDesc array the caller keeps and edits
        in place (no per-call conversion)."""
        self.descs = arr
        check(self._L.axr_batch_set_views(self._h, arr, len(arr)), "axr_batch_set_views")

    def render(self, flags, alpha_index=None, cast=None):
        f = np.ascontiguousarray(np.asarray(flags, np.int32))
        a = None if alpha_index is None else np.ascontiguousarray(np.asarray(alpha_index, np.int32))
        c = None if cast is None else np.ascontiguousarray(np.asarray(cast, np.uint8))
        check(self._L.axr_batch_render(self._h, f.ctypes.data, None if a is None else a.ctypes.data,
                                       None if c is None else c.ctypes.data, len(f)), "axr_batch_render")

    def frame(self, k):
        d = self.descs[k]
        if d.kind == DEPTH:
            m = np.empty((d.w, d.w), np.float32)
            check(self._L.axr_batch_get_frame(self._h, k, None, None, None, m.ctypes.data), "axr_batch_get_frame")
            return m
        r = np.empty((d.h, d.w), np.uint16)
        g = np.empty_like(r)
        b = np.empty_like(r)
        db = np.empty((d.h, d.w), np.float32)
        check(self._L.axr_batch_get_frame(self._h, k, r.ctypes.data, g.ctypes.data, b.ctypes.data, db.ctypes.data),
              "axr_batch_get_frame")
        return r, g, b, db

    def ids(self, k):
        d = self.descs[k]
        t = np.empty((d.h, d.w), np.int32)
        c = np.empty((d.h, d.w), np.uint8)
        check(self._L.axr_batch_get_ids(self._h, k, t.ctypes.data, c.ctypes.data), "axr_batch_get_ids")
        return t, c

    def read_async(self, k, r, g, b, db=None):
        """Queue the copy of shaded view k's planes into host arrays (pinned
        for an asynchronous copy); they hold the data once query() is True."""
        for a in (r, g, b) + ((db,) if db is not None else ()):
            d = self.descs[k]
            assert a.flags.c_contiguous and a.size == d.w * d.h
        check(self._L.axr_batch_read_async(self._h, k, r.ctypes.data, g.ctypes.data, b.ctypes.data,
                                           None if db is None else db.ctypes.data), "axr_batch_read_async")

    def query(self):
        """True once the last render and its read-backs have finished."""
        rc = self._L.axr_batch_query(self._h)
        if rc < 0:
            check(rc, "axr_batch_query")
        return rc == 1

    def phase_times(self):
        """ms of the last render's phases: clear, setup, coarse + small
        triangles + depth maps, tiled large triangles, shading."""
        t = (C.c_float * 5)()
        check(self._L.axr_batch_phase_times(self._h, t), "axr_batch_phase_times")
        return list(t)

    def bytes(self):
        n = C.c_int64()
        check(self._L.axr_batch_bytes(self._h, C.byref(n)), "axr_batch_bytes")
        return n.value

    def set_mode(self, mode):
        """PERSISTENT (one cooperative kernel) or PHASED (one kernel per phase
        in the graph); results are identical."""
        check(self._L.axr_batch_set_mode(self._h, int(mode)), "axr_batch_set_mode")

    def inject_barrier_stall(self, phantom_blocks, spin_limit=1 << 26):
        """Fault injection for failure-detection tests (persistent form): the
        grid barriers of the next renders wait for `phantom_blocks` blocks
        that never run and give up after `spin_limit` polls, so the render
        reports an error instead of hanging.  (0, 1 << 26) restores it."""
        check(self._L.axr_batch_inject_barrier_stall(self._h, int(phantom_blocks), int(spin_limit)),
              "axr_batch_inject_barrier_stall")

    def set_tuning(self, blocks_per_sm, min_chunk):
        check(self._L.axr_batch_set_tuning(self._h, int(blocks_per_sm), int(min_chunk)), "axr_batch_set_tuning")

    def stats(self):
        n, g, gr = C.c_int64(), C.c_int(), C.c_int()
        check(self._L.axr_batch_stats(self._h, C.byref(n), C.byref(g), C.byref(gr)), "axr_batch_stats")
        return {"renders": n.value, "graph": bool(g.value), "grid": gr.value}


def scene_batch_views(scene, main_view, faces_at=None, face_side=512):
    """Depth views for the scene's cascades, then the main view and optional
    cube faces, each shaded view sampling all cascades."""
    descs = [depth(c, scene.bias) for c in scene.shadows]
    casc = list(range(min(2, len(scene.shadows))))
    descs.append(shaded(main_view, casc))
    if faces_at is not None:
        descs += [shaded(v, casc) for v in cube_faces(faces_at, face_side)]
    return descs
