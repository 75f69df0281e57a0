"""CLDraw: drop-in for the reference's draw runtime (PyOpenCL27C/Ops.py:127-1230,
PyOpenCL27C/Ops0.py:93-910), backed by libaxr.so on a B200.

Same method names, argument meanings and return types as the reference's
class, which the engine holds as `ThreeDBackend.draw`
(PyOpenCL27C/Compute.py:182-229,313-339,381-383,426-460).  Differences that
a caller can see:
  - errors raise `AxrError` (the reference raises pyopencl errors)
  - `getIDs()` is new: triangle id and coverage of the last drawAll
  - effects outside the rasterizer hot path (sky, particles, reflections,
    SSR, cubemap re-layout, GI buffers, bones, waves, voxel light, normal
    and roughness maps), the post kernels the snapshot does not ship
    (tonemap, exposure, blurTest) and the OpenCL buffer plumbing
    (getBuffers, getShadow, getArgs) are not provided: their methods raise
    NotImplementedError, except setSkyTex, which the engine calls
    unconditionally and which is accepted and ignored.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import AxrError, check, lib
from .scenes import flags_from_string, view_mat


# sky colour the current reference's clearZBuffer fills the frame with
# (Ops.py:941: (60, 110, 255)^2 / 3 as int32)
SKY_COLOR = tuple(int(x) for x in (np.array([60, 110, 255.0]) ** 2 / 3).astype(np.int32))


def _p(a):
    return None if a is None else a.ctypes.data


def _pad4(v):
    """(V, 3) -> (V // 3, 3, 4) float32 with a zero fourth component
    (the reference's align34 layout, Ops.py:124-125)."""
    out = np.zeros((v.shape[0], 4), np.float32)
    out[:, :3] = v
    return out.reshape(-1, 3, 4)


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


class CLDraw:
    def __init__(self, size_sky, max_uv, w, h, max_particles, device=0, pinned=False):
        self.W, self.H = int(w), int(h)
        self.WC, self.HC = self.W // 16, self.H // 16
        self.LT = max_uv
        self._L = lib()
        h_ = C.c_void_p()
        check(self._L.axr_create(self.W, self.H, int(device), C.byref(h_)), "axr_create")
        self._h = h_
        self.gSize = []           # vertex counts per group (reference name)
        self.texSize = []
        self._mip_bias = []       # mipBias per group, as the library holds it
        self._set_bias = []       # mipBias per group given by setMipBias (0 until set)
        self.NM = {}              # normal maps by name (reference name), library ids
        self._normal = {}         # group -> (map id, roughness, metal) as the library holds it
        self._tex_alpha = 0
        self.SHADOWMAP = {}
        self.ambLight = np.float32(0.2)
        # point and spot lights of vertLight stay set until a call replaces
        # them (None) or clears them (1), as in the reference
        self._points = (np.zeros((0, 3), np.float32),) * 2
        self._spots = (np.zeros((0, 3), np.float32),) * 3
        self._pinned = pinned
        self.hro = self._host((self.H, self.W), np.uint16)
        self.hgo = self._host((self.H, self.W), np.uint16)
        self.hbo = self._host((self.H, self.W), np.uint16)
        self.hdb = self._host((self.H, self.W), np.float32)

    def _host(self, shape, dtype):
        if self._pinned:
            import torch
            t = torch.empty(shape, dtype={np.uint16: torch.uint16, np.float32: torch.float32,
                                          np.int32: torch.int32, np.uint8: torch.uint8}[np.dtype(dtype).type],
                            pin_memory=True)
            self.__dict__.setdefault("_pins", []).append(t)
            return t.numpy()
        return np.ones(shape, dtype)

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                self._L.axr_destroy(self._h)
                self._h = None
        except Exception:
            pass

    # ------------------------------------------------------------ set-up
    def setScaleCull(self, s, cx, cy):
        self.sScale = np.float32(s)
        self.caX, self.caY = np.float32(cx), np.float32(cy)
        check(self._L.axr_set_scale_cull(self._h, float(self.sScale), float(self.caX), float(self.caY)), "setScaleCull")

    def setSkyTex(self, r, g, b, size):
        """Accepted for compatibility; the sky pass is outside this library."""
        self.skyTexSize = np.int32(size)

    def addTextureGroup(self, xyz, uv, vn, r, g, b, mip=False):
        p = _f32(np.asarray(xyz).reshape(-1, 3))
        n = _f32(np.asarray(vn).reshape(-1, 3))
        t = _f32(np.asarray(uv).reshape(-1, 2))
        if p.shape[0] % 3 or n.shape != p.shape or t.shape[0] != p.shape[0]:
            raise AxrError("addTextureGroup: xyz, uv and vn must hold 3 vertices per triangle")
        rr = np.ascontiguousarray(np.asarray(r).astype(np.uint16).reshape(-1))
        gg = np.ascontiguousarray(np.asarray(g).astype(np.uint16).reshape(-1))
        bb = np.ascontiguousarray(np.asarray(b).astype(np.uint16).reshape(-1))
        out = C.c_int()
        check(self._L.axr_add_texture_group(self._h, _p(p), _p(t), _p(n), p.shape[0] // 3, _p(rr), _p(gg), _p(bb),
                                            rr.size, int(mip) if mip else 0, C.byref(out)), "addTextureGroup")
        self.gSize.append(np.int32(p.shape[0]))
        self.texSize.append(np.int32(np.log2(mip)) if mip else np.int32(int(round(rr.size ** 0.5))))
        self._mip_bias.append(np.float32(0.0))
        self._set_bias.append(np.float32(0.0))
        return out.value

    def _apply_mip_bias(self, tn, b):
        if b != self._mip_bias[tn]:
            check(self._L.axr_set_mip_bias(self._h, int(tn), C.c_float(b)), "setMipBias")
            self._mip_bias[tn] = b

    def setMipBias(self, tn, bias):
        """Sets group tn's mipBias (av_draw_normmap_mip.c:43) for the later
        drawAll calls and batch renders whose material for the group carries
        none (new: the reference passes a bias per draw only in its
        normal-mapped mip material, a dict with "normal" and "mip", Ops.py:687,
        797-799; drawAll takes it from such a dict for that draw)."""
        b = np.float32(bias)
        self._set_bias[int(tn)] = b
        self._apply_mip_bias(int(tn), b)

    def setVertLight(self, tn, li):
        """Uploads the per-vertex light `I` of group tn (what vertLight computes)."""
        a = _f32(np.asarray(li).reshape(-1, 3))
        check(self._L.axr_set_vert_light(self._h, int(tn), _p(a)), "setVertLight")

    def vertLight(self, mask, dirI, dirD, pointI=None, pointP=None, spotI=None, spotD=None, spotP=None):
        """Per-vertex light I of every masked group from directional lights
        1.., point and spot lights (vert.c vertL; Ops.py:552-612).  pointI /
        spotI: None keeps the lights of the previous call, 1 clears them,
        arrays [n][3] replace them."""
        def lights(arg, rest, cur):
            if arg is None:
                return cur
            if isinstance(arg, (int, np.integer)) and not isinstance(arg, bool) and arg == 1:
                return tuple(np.zeros((0, 3), np.float32) for _ in cur)
            arrs = tuple(_f32(np.asarray(x).reshape(-1, 3)) for x in (arg, *rest))
            if len({a.shape[0] for a in arrs}) != 1:
                raise ValueError("vertLight: light arrays of different lengths")
            return arrs
        self._points = lights(pointI, (pointP,), self._points)
        self._spots = lights(spotI, (spotD, spotP), self._spots)
        i = _f32(np.asarray(dirI).reshape(-1, 3))
        d = _f32(np.asarray(dirD).reshape(-1, 3))
        m = np.ascontiguousarray(np.asarray(mask, dtype=np.uint8)[:len(self.gSize)])
        if m.size < len(self.gSize):
            raise ValueError("vertLight: mask shorter than the number of groups")
        (pi, pp), (si, sd, sp) = self._points, self._spots
        check(self._L.axr_vert_light(self._h, _p(m), len(self.gSize), _p(i), _p(d), i.shape[0],
                                     _p(pi), _p(pp), pi.shape[0], _p(si), _p(sd), _p(sp), si.shape[0],
                                     float(self.ambLight)), "vertLight")

    def rotate(self, oldRM, rotMat, origin, cStart, cEnd, tn):
        """Rotates vertices [cStart, cEnd) of group tn (None: to the end) about
        origin: p -> rotMat^T (oldRM (p - origin)) + origin, normals alike
        (vert.c transform; Ops.py:481-497)."""
        old = _f32(np.asarray(oldRM).reshape(3, 3))
        rot = _f32(np.asarray(rotMat).reshape(3, 3))
        o = _f32(np.asarray(origin).reshape(3))
        end = -1 if cEnd is None else int(cEnd)
        check(self._L.axr_transform(self._h, int(tn), _p(old), _p(rot), _p(o), int(cStart), end), "rotate")

    def transform(self, oldRM, rotMat, origin, cStart, cEnd, tn):
        """The name VertObject.transform calls (VertObjects.py:238); same as rotate."""
        self.rotate(oldRM, rotMat, origin, cStart, cEnd, tn)

    def translate(self, coords, cStart, cEnd, tn):
        """Moves vertices [cStart, cEnd) of group tn by coords (vert.c
        Ttranslate; Ops.py:499-508)."""
        o = _f32(np.asarray(coords).reshape(3))
        end = -1 if cEnd is None else int(cEnd)
        check(self._L.axr_translate(self._h, int(tn), _p(o), int(cStart), end), "translate")

    def copyTo(self, tn, vp, vn, cstart=0):
        p = _f32(np.asarray(vp).reshape(-1, 3))
        n = _f32(np.asarray(vn).reshape(-1, 3))
        check(self._L.axr_copy_to(self._h, int(tn), _p(p), _p(n), int(cstart), p.shape[0] // 3), "copyTo")

    def getVertices(self, tn):
        """New: group tn's vertex arrays (positions, normals, per-vertex light)
        as (V, 3) float32 host copies, after the work queued before them.
        The reference keeps them in device buffers (getBuffers, Ops.py:618-620)."""
        nv = int(self.gSize[tn])
        out = [np.empty((nv, 3), np.float32) for _ in range(3)]
        check(self._L.axr_get_vertices(self._h, int(tn), *[_p(a) for a in out]), "getVertices")
        return tuple(out)

    def getVertPoints(self, tn):
        """Group tn's positions in the reference's device layout
        (Ops.py:290-293): (T, 3, 4) float32, one float4 per vertex whose
        fourth component is align34's padding, 0."""
        return _pad4(self.getVertices(tn)[0])

    def getVertNorms(self, tn):
        """Group tn's normals in the same layout (Ops.py:294-297)."""
        return _pad4(self.getVertices(tn)[1])

    def addTexAlpha(self, a):
        a = np.asarray(a)
        m = np.ascontiguousarray(a.astype(bool).astype(np.uint8).reshape(-1))
        side = a.shape[0] if a.ndim == 2 else int(round(m.size ** 0.5))
        out = C.c_int()
        check(self._L.axr_add_tex_alpha(self._h, _p(m), side, C.byref(out)), "addTexAlpha")
        return out.value

    def addNrmMap(self, rgb, name, mip=False):
        """CLDraw.addNrmMap(rgb, name) (Ops.py:299-302): an (N, N, 3) uint8
        normal map (or RGBA bytes already laid out, one texel per texel of
        the textures it is used with).  mip=True stores its createMips chain,
        smallest level first, for the normal-mapped mip material."""
        a = np.asarray(rgb)
        if a.ndim == 3:
            from .scenes import create_mips
            flat = create_mips(a[..., :3]) if mip else a[..., :3].reshape(-1, 3)
            out4 = np.zeros((flat.shape[0], 4), np.uint8)
            out4[:, :3] = flat
            a = out4
        b = np.ascontiguousarray(a, np.uint8).reshape(-1)
        if b.size % 4:
            raise AxrError("addNrmMap: expected (N, N, 3) bytes or RGBA bytes")
        out = C.c_int()
        check(self._L.axr_add_normal_map(self._h, _p(b), b.size // 4, C.byref(out)), "addNrmMap")
        self.NM[name] = out.value
        return out.value

    def _draw_normal_materials(self, shaders):
        """The normal-mapped dict materials of one draw ({"normal": (name,
        roughness), "metal": ...}, Ops.py:669-699) to the library."""
        items = shaders.items() if isinstance(shaders, dict) else enumerate(shaders)
        for i, sh in items:
            if not (isinstance(sh, dict) and "normal" in sh):
                continue
            name, rough = sh["normal"][0], sh["normal"][1]
            if name not in self.NM:
                raise AxrError(f"drawAll: normal map {name!r} was not added")
            want = (self.NM[name], float(np.float32(rough)), int("metal" in sh and bool(sh["metal"])))
            if self._normal.get(int(i)) != want:
                check(self._L.axr_set_normal_material(self._h, int(i), want[0], C.c_float(want[1]), want[2]),
                      "setNormalMaterial")
                self._normal[int(i)] = want

    def setPrimaryLight(self, dirI, dirD):
        i = _f32(np.asarray(dirI).reshape(-1, 3)[0])
        d = _f32(np.asarray(dirD).reshape(-1, 3)[0])
        check(self._L.axr_set_primary_light(self._h, _p(i), _p(d)), "setPrimaryLight")

    def setPos(self, vc):
        v = _f32(np.asarray(vc).reshape(3))            # held until the call returns
        check(self._L.axr_set_pos(self._h, _p(v)), "setPos")

    def setVM(self, vM):
        m = _f32(np.asarray(vM)[:3, :3].reshape(9))
        check(self._L.axr_set_vm(self._h, _p(m)), "setVM")

    # ------------------------------------------------------------ frame
    def clearZBuffer(self):
        check(self._L.axr_clear_zbuffer(self._h), "clearZBuffer")

    def clearColor(self, col):
        """Colour half of the current reference's clearZBuffer (Ops.py:939-946):
        fills the colour planes with `col` (three u16 values, e.g. SKY_COLOR)."""
        r, g, b = (int(x) for x in col)
        check(self._L.axr_clear_color(self._h, r, g, b), "clearColor")

    def _material_args(self, shaders):
        n = len(self.gSize)
        if isinstance(shaders, dict):
            shaders = [shaders.get(i, "") for i in range(n)]
        if len(shaders) != n:
            raise AxrError(f"drawAll: {len(shaders)} shaders for {n} groups")
        flags = np.zeros(n, np.int32)
        aidx = np.zeros(n, np.int32)
        for i, s in enumerate(shaders):
            flags[i] = flags_from_string(s)
            if isinstance(s, dict) and "alpha" in s:
                aidx[i] = int(s["alpha"])
        return flags, aidx

    @staticmethod
    def _dict_mip_biases(shaders, n):
        """{group: mipBias} for the dict materials that carry one: the
        reference reads np.float32(material["mip"]) only for its normal-mapped
        mip material, a dict holding both "normal" and "mip" (Ops.py:687,
        797-799); elsewhere "mip" is a flag."""
        items = shaders.items() if isinstance(shaders, dict) else enumerate(shaders)
        return {int(i): np.float32(s["mip"]) for i, s in items
                if isinstance(s, dict) and "mip" in s and "normal" in s and int(i) < n}

    def _draw_mip_biases(self, shaders):
        """Sets every group's mipBias for one draw: its material's, where the
        material carries one, else the setMipBias value (0 until set)."""
        per_draw = self._dict_mip_biases(shaders, len(self.gSize))
        for i in range(len(self.gSize)):
            self._apply_mip_bias(i, per_draw.get(i, self._set_bias[i]))

    def drawAll(self, shaders, mask=None, shadowIds=(0, 1), useOpacitySM=False):
        flags, aidx = self._material_args(shaders)
        self._draw_mip_biases(shaders)
        self._draw_normal_materials(shaders)
        m = None if mask is None else np.ascontiguousarray(np.asarray(mask, dtype=np.uint8))
        ids = [int(i) for i in shadowIds if int(i) in self.SHADOWMAP][:2]
        sid = np.asarray(ids + [0, 0], np.int32)[:2]
        check(self._L.axr_draw_all(self._h, _p(flags), _p(aidx), _p(m), len(flags), _p(sid), len(ids)), "drawAll")

    def getFrame(self):
        check(self._L.axr_get_frame(self._h, _p(self.hro), _p(self.hgo), _p(self.hbo), _p(self.hdb)), "getFrame")
        return (self.hro, self.hgo, self.hbo, self.hdb)

    def readFrameAsync(self):
        """Starts reading the current frame back without waiting (new: the
        reference's getFrame blocks).  Returns a ticket for waitFrame.  The
        frame lands in one of two host buffer sets, reused every second read."""
        if not hasattr(self, "_ring"):
            self._ring = [tuple(self._host((self.H, self.W), t) for t in (np.uint16,) * 3 + (np.float32,))
                          for _ in range(2)]
            self._ring_next = 0
        bufs = self._ring[self._ring_next]
        t = C.c_int64()
        check(self._L.axr_read_frame_async(self._h, *[_p(a) for a in bufs], C.byref(t)), "readFrameAsync")
        self._ring_next ^= 1
        return (t.value, bufs)

    def readFrameRGB8Async(self, ex=1.0):
        """Starts reading the frame back as display-ready 8-bit RGB (H, W, 3):
        Post/gamma.c's mapping with exposure `ex`, packed on the device (new;
        the planes are not changed).  Returns a ticket for waitFrame."""
        if not hasattr(self, "_ring8"):
            self._ring8 = [self._host((self.H, self.W, 3), np.uint8) for _ in range(2)]
            self._ring8_next = 0
        buf = self._ring8[self._ring8_next]
        t = C.c_int64()
        check(self._L.axr_read_frame_rgb8_async(self._h, float(ex), _p(buf), C.byref(t)), "readFrameRGB8Async")
        self._ring8_next ^= 1
        return (t.value, buf)

    def waitFrame(self, ticket):
        """Blocks until the read `ticket` is on the host; returns (r, g, b, depth)."""
        tk, bufs = ticket
        check(self._L.axr_wait_frame(self._h, tk), "waitFrame")
        return bufs

    def frameDone(self, ticket):
        rc = self._L.axr_frame_done(self._h, ticket[0])
        if rc < 0:
            check(rc, "frameDone")
        return rc == 1

    def getIDs(self):
        tid = np.empty((self.H, self.W), np.int32)
        cov = np.empty((self.H, self.W), np.uint8)
        check(self._L.axr_get_ids(self._h, _p(tid), _p(cov)), "getIDs")
        return tid, cov

    def setFrame(self, r=None, g=None, b=None, depth=None):
        arrs = [None if a is None else np.ascontiguousarray(a) for a in (r, g, b, depth)]
        check(self._L.axr_set_frame(self._h, *[_p(a) for a in arrs]), "setFrame")

    def ssao(self, rand=None):
        """Screen-space ambient occlusion on the frame in place (Post/ssao.c;
        Ops.py:973-983).  The random table is drawn once, as the reference
        does (np.random.rand(48)), unless `rand` gives one (>= 32 floats)."""
        if rand is None:
            if getattr(self, "_ssao_rand", None) is None:
                self._ssao_rand = np.random.rand(48).astype(np.float32)
            rand = self._ssao_rand
        t = _f32(np.asarray(rand).reshape(-1))
        check(self._L.axr_ssao(self._h, _p(t), t.size), "ssao")

    def dof(self, focus):
        """Depth-of-field gather on the frame (Post/dof.c; Ops.py:985-995)."""
        check(self._L.axr_dof(self._h, float(np.float32(focus))), "dof")

    def blur(self):
        """The bloom on the frame in place (Post/blur.c + blur2.c; Ops.py:1009-1020)."""
        check(self._L.axr_bloom(self._h), "blur")

    def gamma(self, ex):
        check(self._L.axr_gamma(self._h, float(ex)), "gamma")

    # ------------------------------------------------------------ shadows
    def addShadowMap(self, i, size, scale, ambLight=None, useGI=False):
        if useGI:
            raise NotImplementedError("GI shadow buffers are outside this library")
        if ambLight is not None:
            self.ambLight = np.float32(ambLight)
        check(self._L.axr_add_shadow_map(self._h, int(i), int(size), float(np.float32(scale)),
                                         float(self.ambLight)), "addShadowMap")
        self.SHADOWMAP[int(i)] = {"dim": np.int32(size), "dim2": np.int32(size / 2), "scale": np.float32(scale)}

    def placeShadowMap(self, i, pos, facing, ambLight=None):
        f = _f32(view_mat(*facing))
        p = _f32(np.asarray(pos).reshape(3))
        if ambLight is not None:
            self.ambLight = np.float32(ambLight)
        check(self._L.axr_place_shadow_map(self._h, int(i), _p(p), _p(f.reshape(9)), float(self.ambLight)),
              "placeShadowMap")
        self.SHADOWMAP[int(i)]["vecnp"] = f

    def placeShadowMapBasis(self, i, pos, basis, ambLight=None):
        """placeShadowMap with the 3x3 basis given directly (rows: depth, x, y)."""
        p = _f32(np.asarray(pos).reshape(3))
        f = _f32(np.asarray(basis).reshape(9))
        if ambLight is not None:
            self.ambLight = np.float32(ambLight)
        check(self._L.axr_place_shadow_map(self._h, int(i), _p(p), _p(f), float(self.ambLight)), "placeShadowMap")

    def clearShadowMap(self, i):
        check(self._L.axr_clear_shadow_map(self._h, int(i)), "clearShadowMap")

    def shadowMap(self, i, whichCast, shaders, bias, proj="ortho"):
        if proj != "ortho":
            raise NotImplementedError("only orthographic shadow maps")
        n = len(self.gSize)
        cast = np.ascontiguousarray(np.asarray([bool(c) for c in whichCast], np.uint8))
        flags = np.zeros(n, np.int32)
        aidx = np.zeros(n, np.int32)
        for k in range(n):
            s = shaders[k] if not isinstance(shaders, dict) else shaders.get(k, "")
            if isinstance(s, (bool, int, np.integer)) and not isinstance(s, str):
                # Ops0.shadowMap passes useAlpha: 0 or alpha index + 1
                if int(s):
                    flags[k] = 2
                    aidx[k] = int(s) - 1
            else:
                flags[k] = flags_from_string(s)
                if isinstance(s, dict) and "alpha" in s:
                    aidx[k] = int(s["alpha"])
        check(self._L.axr_shadow_map(self._h, int(i), _p(cast), _p(flags), _p(aidx), n, float(np.float32(bias))),
              "shadowMap")

    def getSHM(self, i):
        d = int(self.SHADOWMAP[int(i)]["dim"])
        out = np.empty((d, d), np.float32)
        check(self._L.axr_get_shadow_map(self._h, int(i), _p(out)), "getSHM")
        return out

    # ------------------------------------------------------------ misc
    def sync(self):
        check(self._L.axr_sync(self._h), "sync")

    def stream_ptr(self) -> int:
        s = C.c_void_p()
        check(self._L.axr_get_stream(self._h, C.byref(s)), "getStream")
        return s.value or 0

    def device_ptrs(self):
        ptrs = [C.c_void_p() for _ in range(5)]
        check(self._L.axr_frame_device_ptrs(self._h, *[C.byref(p) for p in ptrs]), "device_ptrs")
        return [p.value for p in ptrs]

    def lastStats(self):
        vals = [C.c_int64() for _ in range(4)]
        check(self._L.axr_last_stats(self._h, *[C.byref(v) for v in vals]), "lastStats")
        return {"kernels": vals[0].value, "n_small": vals[1].value, "n_large": vals[2].value, "n_units": vals[3].value}

    def launchCount(self) -> int:
        v = C.c_int64()
        check(self._L.axr_launch_count(self._h, C.byref(v)), "launchCount")
        return v.value

    def setShadowMode(self, mode, slice=0):
        """0 (default): one work item per caster row chunk; 2 / 1: the tiled
        shadow pass (maps up to 8192 a side), each tile's units front first /
        as binned.  slice: a tile's units per block (0 keeps it).  The maps
        are the same in every mode."""
        check(self._L.axr_set_shadow_mode(self._h, int(mode), int(slice)), "setShadowMode")

    def shadowStats(self, i):
        """Shadow map i's passes: tiled passes whose unit queue overflowed,
        units and queue capacity of the last pass, its opaque and
        alpha-tested casters."""
        v = (C.c_int64 * 5)()
        check(self._L.axr_shadow_stats(self._h, int(i), v, 5), "shadowStats")
        return dict(zip(("overflows", "units", "cap_units", "casters", "casters_alpha"), (int(x) for x in v)))

    def shadowOverflows(self):
        """Per shadow map (in index order): (overflowed passes, units of the
        last pass, queue capacity)."""
        return [tuple(self.shadowStats(i)[k] for k in ("overflows", "units", "cap_units"))
                for i in sorted(self.SHADOWMAP)]

    def lastQueues(self):
        """Work queues of the last drawAll by kind."""
        v = (C.c_int64 * 5)()
        check(self._L.axr_last_queues(self._h, v, 5), "lastQueues")
        return dict(zip(("small", "small_alpha", "large", "units", "units_alpha"), (int(x) for x in v)))

    def setKernelTiming(self, on=True):
        check(self._L.axr_set_kernel_timing(self._h, 1 if on else 0), "setKernelTiming")

    def kernelTimes(self):
        """{kernel name: (total device ms, launches)} since timing was enabled."""
        mx, nl = 64, 48
        names = C.create_string_buffer(mx * nl)
        ms = (C.c_double * mx)()
        cnt = (C.c_int64 * mx)()
        n = C.c_int()
        check(self._L.axr_kernel_times(self._h, mx, names, nl, ms, cnt, C.byref(n)), "kernelTimes")
        out = {}
        for k in range(n.value):
            nm = names.raw[k * nl:(k + 1) * nl].split(b"\0", 1)[0].decode()
            out[nm] = (ms[k], cnt[k])
        return out

    def __getattr__(self, name):
        if name in ("addTexture", "setReflTex", "setHostSkyTex", "addBoneWeights", "initBoneTransforms",
                    "setBoneTransform", "boneTransform", "setupWave", "updateWave",
                    "highlight", "drawDirectional", "getGIM", "addOpacityMap", "clearShadowOpMap",
                    "shadowClouds", "shadowCloudsOpacity", "tonemap", "mipShadowMap", "setPSTex", "drawPS",
                    "getBoneWeights", "initBoneOrigin", "invbt", "genVoxels",
                    "getVoxels", "voxCopy", "voxLight", "voxTerrain"):
            raise NotImplementedError(f"CLDraw.{name} belongs to an effect outside the rasterizer hot path")
        if name == "addRghMap":
            raise NotImplementedError("CLDraw.addRghMap: only the normal_mip dispatch passes a roughness map "
                                      "(Ops.py:683), and its kernel source av_draw_normmap_mip.c takes none")
        if name in ("exposure", "blurTest"):
            raise NotImplementedError(f"CLDraw.{name} runs a kernel file the reference snapshot does not ship")
        if name in ("getBuffers", "getShadow", "getArgs"):
            raise NotImplementedError(f"CLDraw.{name} hands out OpenCL buffers; this library keeps its buffers "
                                      "on the device behind the C ABI")
        raise AttributeError(name)


# ---------------------------------------------------------------- scene helper

class SceneRenderer:
    """Loads a scenes.Scene into a CLDraw and renders views of it."""

    def __init__(self, scene, w, h, device=0, pinned=False):
        self.scene = scene
        self.draw = CLDraw(1, 64, w, h, 1, device=device, pinned=pinned)
        for g in scene.groups:
            r, gg, b = g.tex
            mip = (1 << g.tex_size) if g.flags & 1 else False
            self.draw.addTextureGroup(g.xyz, g.uv, g.vn, r, gg, b, mip=mip)
        for k, g in enumerate(scene.groups):
            self.draw.setVertLight(k, g.li)
        for m, side in scene.alphas:
            self.draw.addTexAlpha(np.asarray(m).reshape(side, side))
        self.draw.setPrimaryLight(np.asarray(scene.lint)[None], np.asarray(scene.ldir)[None])
        self.draw.ambLight = np.float32(scene.amb)
        for k, sc in enumerate(scene.shadows):
            self.draw.addShadowMap(k, sc.dim, sc.scale, scene.amb)
            self.draw.placeShadowMapBasis(k, sc.pos, sc.vv, scene.amb)
        self.flags = [g.flags for g in scene.groups]
        names = (("mip", 1), ("shadow", 4), ("cull", 8), ("multi", 16))
        for k, g in enumerate(scene.groups):
            if g.mip_bias:
                self.draw.setMipBias(k, g.mip_bias)
        # the mipBias goes through setMipBias; a dict's "mip" is a flag,
        # except in the normal-mapped mip material, which carries its bias
        self.shaders = [{"alpha": g.alpha_index, **{k: 1 for k, b in names if g.flags & b}} if g.flags & 2 else
                        " ".join(k for k, b in names if g.flags & b)
                        for g in scene.groups]
        for k, g in enumerate(scene.groups):
            if g.flags & 32:              # scenes.NORMAL
                self.draw.addNrmMap(g.nm, f"group{k}")
                sh = {"normal": (f"group{k}", g.roughness), **{n: 1 for n, b in names if g.flags & b}}
                if g.flags & 2:
                    sh["alpha"] = g.alpha_index
                if g.metal:
                    sh["metal"] = 1
                if g.flags & 1:
                    sh["mip"] = np.float32(g.mip_bias)
                self.shaders[k] = sh

    def shadow_pass(self):
        for k in range(len(self.scene.shadows)):
            self.draw.clearShadowMap(k)
            self.draw.shadowMap(k, [g.cast for g in self.scene.groups], self.shaders, self.scene.bias)

    def set_view(self, view):
        self.draw.setScaleCull(view.sscale, view.cax, view.cay)
        self.draw.setPos(view.pos)
        self.draw.setVM(view.vv)

    def frame(self, view, shadows=True):
        """shadow maps, clear, drawAll (the per-frame hot path)."""
        if shadows:
            self.shadow_pass()
        self.set_view(view)
        self.draw.clearZBuffer()
        self.draw.drawAll(self.shaders, shadowIds=list(range(min(2, len(self.scene.shadows)))))
