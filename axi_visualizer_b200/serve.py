"""Serving loop: render requests of mixed resolution and scene against scenes
kept resident on the device, with continuous batching.

The reference renders one view per frame from its engine loop
(PyOpenCL27C/Compute.py:313-339 `ThreeDBackend.render` -> `Ops.CLDraw.drawAll`)
and has no request server; this module is the serving form of that draw path.

  * Resident scenes.  All scenes live in ONE draw handle as consecutive group
    ranges (meshes, textures, alpha masks); each scene's two shadow cascades
    are rendered once into the handle's shadow maps and stay resident.  A
    view draws only its scene's group range and counts triangle ids from the
    range's first triangle, so a request renders exactly as it would in a
    handle holding its scene alone.
  * Slabs.  A slab is one batch (axr_batch_*) with a fixed set of view slots
    of the served resolutions.  A launch renders every occupied slot of a slab
    in one persistent cooperative kernel replayed from a captured CUDA graph;
    unoccupied slots are AXR_VIEW_SKIP.  Results are copied back to pinned
    host memory on the slab's copy stream, overlapping later launches.
  * Admission by free HBM.  Slabs are allocated on demand while the resident
    assets plus all slabs stay within the HBM budget; a request is admitted
    when it gets a free slot of its resolution, otherwise it waits.
  * Continuous batching.  Each tick the scheduler retires finished slabs,
    admits waiting requests into idle slabs and launches idle slabs that hold
    requests while fewer than `depth` slabs are in flight.  Requests that
    arrive while others are on the GPU join the next launch; launches queue
    back to back on the device while earlier results are copied back.
  * Host-side failure handling: requests that can never be served are
    rejected, a failed slab allocation is retried on a later tick, requests
    can be cancelled before or after launch, and a slab that does not finish
    within `stall_timeout` fails its requests and is retired.

The scheduler (`Server`) only talks to a backend object, so its logic runs on
the CPU with a fake backend; `GpuBackend` is the CUDA one.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import scenes as S

RESOLUTIONS = ((640, 360), (1280, 720), (1920, 1080), (2560, 1440))
RES_PROBS = (0.4, 0.3, 0.2, 0.1)
# view slots of one slab, by resolution (about the request mix)
DEFAULT_LAYOUT = {(640, 360): 4, (1280, 720): 3, (1920, 1080): 2, (2560, 1440): 1}
HBM_BUDGET = 150e9
FOV = 70.0
# every request starts from a frame filled with the sky colour (the colour
# half of the current reference's clearZBuffer), so its result does not
# depend on what its slot held before
SKY = (1200, 4033, 21675)


@dataclass
class Request:
    rid: int
    scene: int
    w: int
    h: int
    pos: tuple
    target: tuple
    arrival: float                      # seconds from the start of the run
    admitted: float = math.nan
    launched: float = math.nan
    done: float = math.nan
    status: str = "new"                 # queued, admitted, launched, done, rejected, cancelled, failed
    error: str | None = None
    frame: tuple | None = None          # (r, g, b, depth) copies, when the server keeps frames
    launch_id: int = -1

    @property
    def latency(self):
        return self.done - self.arrival

    def view(self):
        return S.View.perspective(self.w, self.h, self.pos, self.target, FOV)


def random_pose(rng, extent=30.0):
    """A camera on a ring around the scene, looking at a point near its centre."""
    a = rng.uniform(0, 2 * math.pi)
    r = rng.uniform(0.5, 1.2) * extent
    pos = (r * math.cos(a), rng.uniform(3.0, 15.0), r * math.sin(a))
    target = (rng.uniform(-5, 5), 0.0, rng.uniform(-5, 5))
    return pos, target


def poisson_trace(n, rate, nscenes, seed=0, resolutions=RESOLUTIONS, probs=RES_PROBS, burst=False):
    """n requests with exponential inter-arrival times of mean 1/rate (all at
    t=0 when burst), uniform scene ids and resolutions drawn with `probs`."""
    rng = np.random.default_rng(seed)
    t = np.zeros(n) if burst else np.cumsum(rng.exponential(1.0 / rate, n))
    scene = rng.integers(0, nscenes, n)
    res = rng.choice(len(resolutions), n, p=np.asarray(probs, float) / np.sum(probs))
    out = []
    for i in range(n):
        pos, target = random_pose(rng)
        w, h = resolutions[res[i]]
        out.append(Request(i, int(scene[i]), int(w), int(h), pos, target, float(t[i])))
    return out


def percentile(x, q):
    return float(np.percentile(np.asarray(x, float), q)) if len(x) else math.nan


# ---------------------------------------------------------------------------
# scheduler
# ---------------------------------------------------------------------------

@dataclass
class Slab:
    sid: int
    slots: list                         # (w, h) per slot
    nbytes: int
    handle: object = None
    state: str = "idle"                 # idle, inflight, retired
    assigned: dict = field(default_factory=dict)   # slot -> Request
    launched_at: float = math.nan
    launches: int = 0
    solo: bool = False                  # one slot: takes a request that arrives alone

    def free_slot(self, w, h):
        for k, wh in enumerate(self.slots):
            if wh == (w, h) and k not in self.assigned:
                return k
        return None


class Server:
    """Continuous-batching request scheduler over a slab backend.

    backend: create(slots) -> handle, slab_bytes(slots) -> int,
             launch(handle, {slot: Request}), poll(handle) -> bool,
             result(handle, slot) -> (r, g, b, depth), destroy(handle),
             scenes -> number of resident scenes.
    """

    def __init__(self, backend, budget_bytes=HBM_BUDGET, resident_bytes=0, layout=None, max_slabs=8, depth=2,
                 stall_timeout=10.0, keep_frames=False, retry_after=0.05):
        self.b = backend
        self.layout = dict(layout or DEFAULT_LAYOUT)
        self.slot_list = [wh for wh, n in self.layout.items() for _ in range(n)]
        self.slab_bytes = int(backend.slab_bytes(self.slot_list))
        self.budget = float(budget_bytes)
        self.resident = int(resident_bytes)
        self.used = self.resident
        self.peak = self.used
        self.max_slabs, self.depth = int(max_slabs), int(depth)
        self.stall_timeout, self.keep_frames, self.retry_after = stall_timeout, keep_frames, retry_after
        # waiting requests, first come first served per resolution (a slot
        # only ever takes requests of its own resolution)
        self.queues: dict[tuple, deque] = {wh: deque() for wh in self.layout}
        self.slabs: list[Slab] = []
        self.requests: dict[int, Request] = {}
        self.launch_sizes: list[int] = []
        self.max_inflight = 0
        self.alloc_failures = 0
        self.low_memory = 0
        self.hbm_reserve = 1 << 30        # free HBM kept back when making a slab
        self._next_alloc = -math.inf
        self._sid = 0

    # -- requests
    def submit(self, req: Request, now: float):
        self.requests[req.rid] = req
        if req.scene < 0 or req.scene >= self.b.scenes:
            return self._reject(req, f"scene {req.scene} is not resident")
        if (req.w, req.h) not in self.layout:
            return self._reject(req, f"resolution {req.w}x{req.h} is not served")
        if self.resident + self.slab_bytes > self.budget:
            return self._reject(req, "a slab does not fit in the HBM budget")
        req.status = "queued"
        self.queues[(req.w, req.h)].append(req)

    def cancel(self, rid: int):
        """Cancels a request: a queued or admitted one is dropped before launch;
        the result of a launched one is discarded."""
        r = self.requests.get(rid)
        if r is None or r.status in ("done", "rejected", "cancelled", "failed"):
            return False
        if r.status == "queued":
            self.queues[(r.w, r.h)].remove(r)
        elif r.status == "admitted":
            for s in self.slabs:
                for k, q in list(s.assigned.items()):
                    if q is r and s.state == "idle":
                        del s.assigned[k]
        r.status = "cancelled"
        return True

    def _reject(self, req, why):
        req.status, req.error = "rejected", why

    # -- one tick
    def step(self, now: float):
        self._retire(now)
        self._admit(now)
        self._launch(now)

    def _retire(self, now):
        for s in self.slabs:
            if s.state == "inflight" and self.b.poll(s.handle):
                for k, r in s.assigned.items():
                    if r.status == "cancelled":
                        continue
                    if self.keep_frames:
                        r.frame = tuple(np.array(a, copy=True) for a in self.b.result(s.handle, k))
                    r.done, r.status = now, "done"
                s.assigned.clear()
                s.state = "idle"
            elif s.state == "inflight" and now - s.launched_at > self.stall_timeout:
                for r in s.assigned.values():
                    if r.status != "cancelled":
                        r.status, r.error, r.done = "failed", "render stalled", now
                s.assigned.clear()
                s.state = "retired"      # never reused; released once it completes
        for s in [s for s in self.slabs if s.state == "retired"]:
            if self.b.poll(s.handle):
                self.b.destroy(s.handle)
                self.slabs.remove(s)
                self.used -= s.nbytes

    def prepare(self, n):
        """Makes up to n slabs ahead of the first request (as the budget
        allows), so that no request waits for a slab to be made."""
        while len(self.slabs) < min(n, self.max_slabs) and self._new_slab(-math.inf, force=True):
            pass
        return len(self.slabs)

    def prepare_solo(self):
        """Makes one single-slot slab per served resolution (as the budget
        allows): a request that arrives while nothing renders and nothing
        else waits is launched there, without the other slots of a full
        slab."""
        for wh in self.layout:
            if not any(s.solo and s.slots[0] == wh for s in self.slabs):
                self._new_slab(-math.inf, force=True, slots=[wh])
        return sum(1 for s in self.slabs if s.solo)

    def _new_slab(self, now, force=False, slots=None):
        solo = slots is not None
        slots = list(slots) if solo else list(self.slot_list)
        nbytes = int(self.b.slab_bytes(slots)) if solo else self.slab_bytes
        if not solo and len([s for s in self.slabs if s.state != "retired" and not s.solo]) >= self.max_slabs:
            return None
        if self.used + nbytes > self.budget or (now < self._next_alloc and not force):
            return None
        free = getattr(self.b, "free_bytes", None)
        if free is not None and free() < nbytes + self.hbm_reserve:
            self.low_memory += 1          # the device has less free HBM than the budget assumed
            return None
        try:
            h = self.b.create(slots)
        except (MemoryError, RuntimeError) as e:   # AxrError is a RuntimeError
            self.alloc_failures += 1
            self._next_alloc = now + self.retry_after
            self.last_alloc_error = str(e)
            return None
        s = Slab(self._sid, slots, nbytes, h, solo=solo)
        self._sid += 1
        self.slabs.append(s)
        self.used += s.nbytes
        self.peak = max(self.peak, self.used)
        return s

    def _fill(self, s, now):
        if s.solo:
            return
        for k, wh in enumerate(s.slots):
            q = self.queues[wh]
            if q and k not in s.assigned:
                r = q.popleft()
                s.assigned[k] = r
                r.status, r.admitted = "admitted", now

    def _admit(self, now):
        """Free slots of idle slabs take the oldest waiting request of their
        resolution; while requests still wait, new slabs are made as the
        budget allows.  A request that waits alone while nothing renders
        goes to an idle single-slot slab of its resolution, if there is one."""
        waiting = [q for q in self.queues.values() if q]
        if len(waiting) == 1 and len(waiting[0]) == 1 and not any(s.state == "inflight" for s in self.slabs) \
                and not any(s.assigned for s in self.slabs):
            r = waiting[0][0]
            solo = next((s for s in self.slabs if s.solo and s.state == "idle" and s.slots[0] == (r.w, r.h)), None)
            if solo is not None:
                waiting[0].popleft()
                solo.assigned[0] = r
                r.status, r.admitted = "admitted", now
                return
        for s in self.slabs:
            if s.state == "idle":
                self._fill(s, now)
        if any(self.queues.values()):
            # at most one new slab per tick: what it costs (allocation, pinned
            # host buffers, graph capture) must not hold back launches
            s = self._new_slab(now)
            if s is not None:
                self._fill(s, now)

    def _launch(self, now):
        inflight = sum(1 for s in self.slabs if s.state == "inflight")
        ready = [s for s in self.slabs if s.state == "idle" and s.assigned]
        ready.sort(key=lambda s: min(r.arrival for r in s.assigned.values()))
        for s in ready:
            if inflight >= self.depth:
                break
            self.b.launch(s.handle, dict(s.assigned))
            s.state, s.launched_at = "inflight", now
            s.launches += 1
            lid = len(self.launch_sizes)
            self.launch_sizes.append(len(s.assigned))
            for r in s.assigned.values():
                r.status, r.launched, r.launch_id = "launched", now, lid
            inflight += 1
        self.max_inflight = max(self.max_inflight, inflight)

    def reset_stats(self):
        """Forgets finished requests and launch records (slabs stay warm)."""
        self.requests = {k: r for k, r in self.requests.items() if r.status in ("queued", "admitted", "launched")}
        self.launch_sizes = []
        self.max_inflight = 0
        self.peak = self.used

    def close(self):
        """Waits for the slabs in flight and releases every slab."""
        for s in self.slabs:
            while s.state == "inflight" and not self.b.poll(s.handle):
                time.sleep(1e-4)
            self.b.destroy(s.handle)
            self.used -= s.nbytes
        self.slabs = []

    # -- driving
    def busy(self):
        return any(self.queues.values()) or any(s.state == "inflight" or s.assigned for s in self.slabs)

    def run(self, trace, clock=time.perf_counter, poll=0.0, timeout=600.0):
        """Feeds `trace` in real time (arrival offsets from the start) and ticks
        until every request has finished (polling every `poll` s while work is
        on the GPU; 0 spins, yielding the processor).  Returns stats()."""
        trace = sorted(trace, key=lambda r: r.arrival)
        t0 = clock()
        i = 0
        while i < len(trace) or self.busy():
            now = clock() - t0
            while i < len(trace) and trace[i].arrival <= now:
                self.submit(trace[i], now)
                i += 1
            self.step(now)
            if now > timeout:
                raise TimeoutError("serving run did not finish")
            if not self.busy() and i < len(trace):
                time.sleep(max(0.0, min(trace[i].arrival - now, 0.002)))
            else:
                time.sleep(poll)
        self.wall = clock() - t0
        return self.stats(trace)

    def stats(self, trace):
        done = [r for r in trace if r.status == "done"]
        lat = [r.latency * 1e3 for r in done]
        span = (max(r.done for r in done) - min(r.arrival for r in trace)) if done else math.nan
        px = sum(r.w * r.h for r in done)
        return {
            "requests": len(trace), "done": len(done),
            "rejected": sum(r.status == "rejected" for r in trace),
            "cancelled": sum(r.status == "cancelled" for r in trace),
            "failed": sum(r.status == "failed" for r in trace),
            "frames_per_s": len(done) / span if done else 0.0,
            "Mpix_per_s": px / span / 1e6 if done else 0.0,
            "p50_ms": percentile(lat, 50), "p99_ms": percentile(lat, 99), "max_ms": max(lat) if lat else math.nan,
            "launches": len(self.launch_sizes),
            "views_per_launch": float(np.mean(self.launch_sizes)) if self.launch_sizes else 0.0,
            "max_inflight": self.max_inflight,
            "slabs": len(self.slabs), "slab_bytes": self.slab_bytes,
            "hbm_used_peak_bytes": self.peak, "hbm_budget_bytes": self.budget, "resident_bytes": self.resident,
            "alloc_failures": self.alloc_failures, "low_memory_skips": self.low_memory,
        }


# ---------------------------------------------------------------------------
# resident scenes and the CUDA backend
# ---------------------------------------------------------------------------

def _shader(g, alpha_base):
    """CLDraw shader description of a scenes.Group (alpha index made global;
    the group's mipBias is set with setMipBias, a dict's "mip" is a flag)."""
    names = [k for k, b in (("mip", 1), ("shadow", 4), ("cull", 8)) if g.flags & b]
    if g.flags & 2:
        return {"alpha": alpha_base + g.alpha_index, **{k: 1 for k in names}}
    return " ".join(names)


def load_scenes(draw, scenes):
    """Adds every scene's groups, alpha masks and shadow cascades to one
    CLDraw and renders the cascades.  Returns per scene a dict with its group
    range, shadow-map ids and triangle count, and the global shader list."""
    info, shaders, group = [], [], 0
    alpha_base = 0
    light = None
    for si, sc in enumerate(scenes):
        key = (tuple(np.asarray(sc.lint, np.float32)), tuple(np.asarray(sc.ldir, np.float32)), float(sc.amb))
        if light is None:
            light = key
            draw.setPrimaryLight(np.asarray(sc.lint)[None], np.asarray(sc.ldir)[None])
            draw.ambLight = np.float32(sc.amb)
        elif key != light:
            raise ValueError(f"scene {si}: resident scenes share one sun and ambient term")
        first = group
        for g in sc.groups:
            r, gg, b = g.tex
            draw.addTextureGroup(g.xyz, g.uv, g.vn, r, gg, b, mip=(1 << g.tex_size) if g.flags & 1 else False)
            draw.setVertLight(group, g.li)
            if g.mip_bias:
                draw.setMipBias(group, g.mip_bias)
            shaders.append(_shader(g, alpha_base))
            group += 1
        for m, side in sc.alphas:
            draw.addTexAlpha(np.asarray(m).reshape(side, side))
        alpha_base += len(sc.alphas)
        ids = []
        for cam in sc.shadows[:2]:
            k = len(draw.SHADOWMAP)
            draw.addShadowMap(k, cam.dim, cam.scale, sc.amb)
            draw.placeShadowMapBasis(k, cam.pos, cam.vv, sc.amb)
            ids.append(k)
        info.append({"groups": (first, len(sc.groups)), "shadows": ids, "bias": float(sc.bias),
                     "tris": sum(len(g.xyz) // 3 for g in sc.groups), "cast": [bool(g.cast) for g in sc.groups]})
    for si, d in enumerate(info):
        first, n = d["groups"]
        cast = [False] * group
        for g in range(n):
            cast[first + g] = d["cast"][g]
        for k in d["shadows"]:
            draw.clearShadowMap(k)
            draw.shadowMap(k, cast, shaders, d["bias"])
    draw.sync()
    return info, shaders


def _device_free(device):
    import torch
    torch.cuda.synchronize(device)
    return torch.cuda.mem_get_info(device)[0]


def _pinned(n, dtype):
    import torch
    t = torch.empty(n, dtype={np.uint16: torch.uint16, np.float32: torch.float32}[dtype], pin_memory=True)
    return t, t.numpy()


class ResidentScenes:
    """Every scene resident in one draw handle; `nbytes` is the device memory
    the handle took (free HBM before minus after loading)."""

    def __init__(self, scenes, device=0):
        from .ops import CLDraw
        self.scenes = list(scenes)
        self.device = device
        free0 = _device_free(device)
        self.draw = CLDraw(1, 64, 64, 64, 1, device=device)
        self.info, self.shaders = load_scenes(self.draw, self.scenes)
        self.flags, self.aidx = self.draw._material_args(self.shaders)
        self.nbytes = int(free0 - _device_free(device))
        self.total_tris = sum(d["tris"] for d in self.info)


MAX_CHUNKS = 8           # small-triangle work items per triangle (kernels.cuh)
CTR_WORDS = 32


class GpuBackend:
    """Slabs as axr_batch objects over a ResidentScenes handle."""

    def __init__(self, resident: ResidentScenes, tuning=None, read_depth=True, mode=1):
        from . import batch as B
        self.B = B
        self.res = resident
        self.scenes = len(resident.scenes)
        self.tuning = tuning
        # batch.PHASED by default: slabs hold heavy views (50k-1M triangles at
        # up to 2560x1440), where one kernel per phase beats the persistent one
        self.mode = mode
        self.read_depth = read_depth

    def free_bytes(self):
        """Free HBM on the device right now (other processes may hold some)."""
        import torch
        return torch.cuda.mem_get_info(self.res.device)[0]

    def slab_bytes(self, slots):
        """Device bytes of a slab: framebuffers (3 x u16 colour, f32 depth,
        u64 visibility word per pixel), per-view triangle lists and unit queue
        (as axr_batch_create allocates them), plus 1 MiB for the tables."""
        cap = max(self.res.total_tris, 1)
        units = 1 << 20
        per_view = 4 * cap * (2 + MAX_CHUNKS) + 8 * units + 4 * CTR_WORDS
        return sum(18 * w * h + per_view for w, h in slots) + (1 << 20)

    def create(self, slots):
        """A slab: its batch (every slot AXR_VIEW_SKIP, rendered once so the
        graph is captured now), its view table and pinned result buffers."""
        skips = [self.B.skip(w, h) for w, h in slots]
        bt = self.B.Batch(self.res.draw, skips)
        if self.mode is not None:
            bt.set_mode(self.mode)
        if self.tuning:
            bt.set_tuning(*self.tuning)
        bt.render(self.res.flags, self.res.aidx)
        bufs, ptrs = [], []
        for w, h in slots:
            t, a = _pinned(4 * w * h, np.uint16)
            d = _pinned(w * h, np.float32) if self.read_depth else (None, None)
            bufs.append((t, a, d))
            n = w * h
            base = a.ctypes.data
            ptrs.append((base, base + 2 * n, base + 4 * n, None if d[1] is None else d[1].ctypes.data))
        arr = (self.B.ViewDesc * len(slots))(*skips)
        return {"batch": bt, "slots": list(slots), "bufs": bufs, "ptrs": ptrs, "arr": arr, "skips": skips,
                "used": set()}

    def descs_for(self, slots, assigned):
        out = []
        for k, (w, h) in enumerate(slots):
            r = assigned.get(k)
            out.append(self.B.skip(w, h) if r is None else self.desc(r))
        return out

    def desc(self, r):
        d = self.res.info[r.scene]
        return self.B.shaded(r.view(), [-1 - i for i in d["shadows"]], groups=d["groups"], clear=SKY)

    def launch(self, h, assigned):
        bt, arr = h["batch"], h["arr"]
        for k in h["used"] - set(assigned):
            arr[k] = h["skips"][k]
        for k, r in assigned.items():
            arr[k] = self.desc(r)
        h["used"] = set(assigned)
        bt.set_views_array(arr)
        bt.render(self.res.flags, self.res.aidx)
        L, bh = bt._L, bt._h
        for k in assigned:
            r, g, b, d = h["ptrs"][k]
            rc = L.axr_batch_read_async(bh, k, r, g, b, d)
            if rc:
                self.B.check(rc, "axr_batch_read_async")

    def poll(self, h):
        return h["batch"].query()

    def result(self, h, k):
        w, hh = h["slots"][k]
        n = w * hh
        _, a, (_, d) = h["bufs"][k]
        rgb = tuple(a[i * n:(i + 1) * n].reshape(hh, w) for i in range(3))
        return rgb + ((d.reshape(hh, w),) if d is not None else (None,))

    def destroy(self, h):
        h["batch"]._L.axr_batch_destroy(h["batch"]._h)
        h["batch"]._h = None


# ---------------------------------------------------------------------------
# the plain per-view path on the same trace
# ---------------------------------------------------------------------------

class PlainServer:
    """First-come first-served through the plain per-view path: one CLDraw per
    resolution holding every scene; each request is one drawAll over its
    scene's groups (the others masked) followed by getFrame."""

    def __init__(self, scenes, resolutions, device=0, pinned=True):
        from .ops import CLDraw
        self.draws = {}
        for w, h in resolutions:
            d = CLDraw(1, 64, w, h, 1, device=device, pinned=pinned)
            info, shaders = load_scenes(d, scenes)
            self.draws[(w, h)] = (d, info, shaders)

    def render(self, r: Request):
        d, info, shaders = self.draws[(r.w, r.h)]
        s = info[r.scene]
        first, n = s["groups"]
        mask = [0 if first <= g < first + n else 1 for g in range(len(shaders))]
        v = r.view()
        d.setScaleCull(v.sscale, v.cax, v.cay)
        d.setPos(v.pos)
        d.setVM(v.vv)
        d.clearZBuffer()
        d.clearColor(SKY)
        d.drawAll(shaders, mask=mask, shadowIds=s["shadows"])
        return d.getFrame()

    def run(self, trace, clock=time.perf_counter, keep_frames=False):
        trace = sorted(trace, key=lambda r: r.arrival)
        t0 = clock()
        for r in trace:
            now = clock() - t0
            if r.arrival > now:
                time.sleep(r.arrival - now)
            r.admitted = r.launched = clock() - t0
            f = self.render(r)
            if keep_frames:
                r.frame = tuple(np.array(a, copy=True) for a in f)
            r.done, r.status = clock() - t0, "done"
        done = [r for r in trace if r.status == "done"]
        lat = [r.latency * 1e3 for r in done]
        span = max(r.done for r in done) - min(r.arrival for r in trace)
        return {"requests": len(trace), "done": len(done), "frames_per_s": len(done) / span,
                "Mpix_per_s": sum(r.w * r.h for r in done) / span / 1e6,
                "p50_ms": percentile(lat, 50), "p99_ms": percentile(lat, 99), "max_ms": max(lat)}
