"""Serving scheduler on the CPU with a fake slab backend: request trace,
continuous batching, admission against the HBM budget, rejection, allocation
failure and retry, cancellation, and a stalled render (all failures injected
on the host)."""
import math

import numpy as np
import pytest

from axi_visualizer_b200 import serve as SV

RES = ((64, 32), (128, 64))


class FakeBackend:
    """Slabs whose renders finish after `complete_after` polls; `stall` makes
    the next created slab never finish until released."""

    scenes = 3

    def __init__(self, complete_after=1, fail_creates=0):
        self.complete_after = complete_after
        self.fail_creates = fail_creates
        self.stall_next = False
        self.created, self.destroyed, self.launches = [], [], []

    def slab_bytes(self, slots):
        return 100 * len(slots)

    def create(self, slots):
        if self.fail_creates > 0:
            self.fail_creates -= 1
            raise MemoryError("injected allocation failure")
        h = {"slots": list(slots), "polls": 0, "assigned": {}, "stall": self.stall_next}
        self.stall_next = False
        self.created.append(h)
        return h

    def launch(self, h, assigned):
        h["assigned"], h["polls"] = dict(assigned), 0
        self.launches.append(sorted(r.rid for r in assigned.values()))

    def poll(self, h):
        h["polls"] += 1
        return not h["stall"] and h["polls"] > self.complete_after

    def result(self, h, k):
        r = h["assigned"][k]
        return tuple(np.full((r.h, r.w), r.rid, np.uint16) for _ in range(3)) + (np.zeros((r.h, r.w), np.float32),)

    def destroy(self, h):
        self.destroyed.append(h)


def req(rid, scene=0, res=RES[0], t=0.0):
    return SV.Request(rid, scene, res[0], res[1], (0, 5, -20), (0, 0, 0), t)


def drive(srv, until, t=0.0, dt=0.01):
    while srv.busy() and t < until:
        srv.step(t)
        t += dt
    return t


def test_poisson_trace_statistics():
    tr = SV.poisson_trace(20000, 200.0, 8, seed=4)
    gaps = np.diff([r.arrival for r in tr])
    assert abs(gaps.mean() - 1 / 200) < 0.03 / 200
    assert abs(gaps.std() - 1 / 200) < 0.05 / 200          # exponential: sd == mean
    counts = {wh: 0 for wh in SV.RESOLUTIONS}
    for r in tr:
        counts[(r.w, r.h)] += 1
    for wh, p in zip(SV.RESOLUTIONS, SV.RES_PROBS):
        assert abs(counts[wh] / len(tr) - p) < 0.015
    assert {r.scene for r in tr} == set(range(8))
    again = SV.poisson_trace(20000, 200.0, 8, seed=4)
    assert [(r.arrival, r.scene, r.w, r.pos) for r in tr[:50]] == [(r.arrival, r.scene, r.w, r.pos) for r in again[:50]]
    burst = SV.poisson_trace(10, 200.0, 8, seed=4, burst=True)
    assert all(r.arrival == 0.0 for r in burst)


def test_continuous_batching_joins_next_launch():
    be = FakeBackend(complete_after=2)
    srv = SV.Server(be, budget_bytes=1e9, layout={RES[0]: 2, RES[1]: 1}, max_slabs=2, depth=1, keep_frames=True)
    srv.submit(req(0), 0.0)
    srv.step(0.0)
    assert be.launches == [[0]]                            # launched at once: nothing else on the GPU
    for i, res in ((1, RES[0]), (2, RES[1]), (3, RES[0])):   # exactly one free slab's slots
        srv.submit(req(i, res=res), 0.001)
    srv.step(0.001)                                        # first slab still in flight
    assert be.launches == [[0]]
    assert {srv.requests[i].status for i in (1, 2, 3)} == {"admitted"}
    drive(srv, 1.0, 0.002)
    assert be.launches == [[0], [1, 2, 3]]                 # the arrivals shared the next launch
    for i in range(4):
        r = srv.requests[i]
        assert r.status == "done" and r.frame[0][0, 0] == i and r.frame[0].shape == (r.h, r.w)
    st = srv.stats([srv.requests[i] for i in range(4)])
    assert st["done"] == 4 and st["launches"] == 2 and st["views_per_launch"] == 2.0


def test_pipeline_depth_overlaps_slabs():
    be = FakeBackend(complete_after=3)
    srv = SV.Server(be, budget_bytes=1e9, layout={RES[0]: 1}, max_slabs=4, depth=2)
    for i in range(6):
        srv.submit(req(i), 0.0)
    srv.step(0.0)
    assert len(be.launches) == 1 and len(be.created) == 1   # one new slab per tick
    srv.step(0.001)
    assert len(be.launches) == 2 and srv.max_inflight == 2  # two launches queued back to back
    drive(srv, 5.0)
    assert all(srv.requests[i].status == "done" for i in range(6))
    assert srv.max_inflight == 2


def test_prepare_makes_slabs_ahead_within_budget():
    be = FakeBackend()
    slab = be.slab_bytes([RES[0]])
    srv = SV.Server(be, budget_bytes=3 * slab + 10, layout={RES[0]: 1}, max_slabs=8)
    assert srv.prepare(8) == 3 and len(be.created) == 3     # the budget holds three
    for i in range(3):
        srv.submit(req(i), 0.0)
    srv.step(0.0)
    assert len(be.launches) == 2 and len(be.created) == 3   # depth 2, no new slab needed
    drive(srv, 1.0)
    assert all(srv.requests[i].status == "done" for i in range(3))


def test_admission_respects_hbm_budget():
    be = FakeBackend(complete_after=1)
    slab = be.slab_bytes([RES[0]] * 2)
    resident = 1000
    srv = SV.Server(be, budget_bytes=resident + slab + 50, resident_bytes=resident, layout={RES[0]: 2}, max_slabs=8)
    for i in range(7):
        srv.submit(req(i), 0.0)
    srv.step(0.0)
    assert len(be.created) == 1                            # a second slab would pass the budget
    assert sum(r.status == "queued" for r in srv.requests.values()) == 5
    drive(srv, 5.0)
    assert all(r.status == "done" for r in srv.requests.values())
    assert srv.peak <= srv.budget and len(be.created) == 1
    assert be.launches == [[0, 1], [2, 3], [4, 5], [6]]


def test_rejects_what_can_never_be_served():
    be = FakeBackend()
    srv = SV.Server(be, budget_bytes=1e9, layout={RES[0]: 1})
    srv.submit(req(0, scene=7), 0.0)
    srv.submit(req(1, res=(32, 32)), 0.0)
    srv.submit(req(2), 0.0)
    drive(srv, 1.0)
    st = [srv.requests[i].status for i in range(3)]
    assert st == ["rejected", "rejected", "done"]
    assert "not resident" in srv.requests[0].error and "not served" in srv.requests[1].error
    tiny = SV.Server(FakeBackend(), budget_bytes=10, resident_bytes=5, layout={RES[0]: 1})
    tiny.submit(req(0), 0.0)
    assert tiny.requests[0].status == "rejected" and "budget" in tiny.requests[0].error


def test_admission_checks_free_device_memory():
    """Besides the budget, a slab is made only while the device reports
    enough free HBM (another process may hold memory)."""
    be = FakeBackend()
    free = {"bytes": 10 ** 12}
    be.free_bytes = lambda: free["bytes"]
    srv = SV.Server(be, budget_bytes=1e9, layout={RES[0]: 1}, max_slabs=4)
    srv.hbm_reserve = 1000
    free["bytes"] = 500                                    # below slab + reserve
    srv.submit(req(0), 0.0)
    srv.step(0.0)
    assert len(be.created) == 0 and srv.requests[0].status == "queued" and srv.low_memory == 1
    free["bytes"] = 10 ** 12
    drive(srv, 1.0, 0.01)
    assert srv.requests[0].status == "done" and len(be.created) == 1


def test_allocation_failure_is_retried():
    be = FakeBackend(fail_creates=2)
    srv = SV.Server(be, budget_bytes=1e9, layout={RES[0]: 1}, retry_after=0.05)
    srv.submit(req(0), 0.0)
    srv.step(0.0)
    assert srv.alloc_failures == 1 and srv.requests[0].status == "queued"
    srv.step(0.01)                                         # inside the back-off: no new attempt
    assert srv.alloc_failures == 1
    drive(srv, 2.0, 0.06)
    assert srv.alloc_failures == 2 and srv.requests[0].status == "done"


def test_cancel_before_and_after_launch():
    be = FakeBackend(complete_after=2)
    srv = SV.Server(be, budget_bytes=1e9, layout={RES[0]: 1}, max_slabs=1, depth=1, keep_frames=True)
    for i in range(3):
        srv.submit(req(i), 0.0)
    srv.step(0.0)
    assert srv.requests[0].status == "launched" and srv.requests[1].status == "queued"
    assert srv.cancel(1) and srv.cancel(0)                 # one queued, one on the GPU
    assert not srv.cancel(0)
    drive(srv, 2.0, 0.001)
    assert [srv.requests[i].status for i in range(3)] == ["cancelled", "cancelled", "done"]
    assert srv.requests[0].frame is None
    assert be.launches == [[0], [2]]


def test_stalled_render_fails_its_requests_and_is_retired():
    be = FakeBackend(complete_after=1)
    be.stall_next = True
    srv = SV.Server(be, budget_bytes=1e9, layout={RES[0]: 1}, max_slabs=2, depth=2, stall_timeout=1.0)
    srv.submit(req(0), 0.0)
    srv.step(0.0)
    srv.step(0.5)
    assert srv.requests[0].status == "launched"
    srv.step(1.5)                                          # past the stall timeout
    assert srv.requests[0].status == "failed" and "stalled" in srv.requests[0].error
    srv.submit(req(1), 1.6)
    drive(srv, 3.0, 1.6)
    assert srv.requests[1].status == "done"
    stalled = be.created[0]
    assert stalled not in be.destroyed                     # still running: not released
    stalled["stall"] = False
    srv.step(3.5)
    assert stalled in be.destroyed and len(srv.slabs) == 1
    assert srv.used == srv.resident + srv.slab_bytes


def test_run_in_real_time_with_fake_backend():
    be = FakeBackend(complete_after=0)
    srv = SV.Server(be, budget_bytes=1e9, layout={wh: 2 for wh in RES})
    tr = SV.poisson_trace(40, 2000.0, 3, seed=1, resolutions=RES, probs=(0.5, 0.5))
    st = srv.run(tr, timeout=30.0)
    assert st["done"] == 40 and st["p99_ms"] >= st["p50_ms"] > 0
    assert math.isfinite(st["frames_per_s"]) and st["frames_per_s"] > 0


def test_slab_bytes_formula():
    class R:
        total_tris = 1000
        scenes = [1]
    be = SV.GpuBackend.__new__(SV.GpuBackend)
    be.res = R()
    n = be.slab_bytes([(640, 360), (1280, 720)])
    per_view = 4 * 1000 * (2 + SV.MAX_CHUNKS) + 8 * (1 << 20) + 128
    assert n == 18 * (640 * 360 + 1280 * 720) + 2 * per_view + (1 << 20)


@pytest.mark.parametrize("bad", [-1, 3])
def test_scene_range_checked(bad):
    srv = SV.Server(FakeBackend(), budget_bytes=1e9, layout={RES[0]: 1})
    srv.submit(req(0, scene=bad), 0.0)
    assert srv.requests[0].status == "rejected"


def test_lone_request_goes_to_a_single_slot_slab():
    """A request that arrives while nothing renders and nothing else waits is
    launched in a one-slot slab of its resolution; requests that overlap
    fill the full slabs as before, and every result is still delivered."""
    be = FakeBackend(complete_after=1)
    srv = SV.Server(be, budget_bytes=10_000, layout={RES[0]: 2, RES[1]: 1}, max_slabs=2, depth=2, keep_frames=True)
    assert srv.prepare(1) == 1 and srv.prepare_solo() == 2
    assert sorted(len(h["slots"]) for h in be.created) == [1, 1, 3]
    srv.submit(req(1, res=RES[1]), 0.0)
    srv.step(0.0)
    solo = [s for s in srv.slabs if s.solo and s.state == "inflight"]
    assert len(solo) == 1 and solo[0].slots == [RES[1]] and be.launches == [[1]]
    drive(srv, 1.0)
    # two requests at once: they share a full slab
    srv.submit(req(2, res=RES[0]), 1.0)
    srv.submit(req(3, res=RES[0]), 1.0)
    srv.step(1.0)
    assert be.launches[-1] == [2, 3]
    assert not any(s.solo and s.state == "inflight" for s in srv.slabs)
    drive(srv, 2.0, t=1.0)
    for rid in (1, 2, 3):
        r = srv.requests[rid]
        assert r.status == "done" and int(r.frame[0][0, 0]) == rid
