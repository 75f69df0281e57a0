"""Autotuner for the batched renderer's scheduling knobs.

Knobs (none of them changes a result; views stay bit-identical):
  mode           persistent (one cooperative kernel, grid barriers between the
                 phases: fewest launches) or phased (one kernel per phase in
                 the graph, each at its own occupancy, alpha-tested work on a
                 parallel branch: better for heavy views)
  blocks_per_sm  size of the persistent cooperative grid (1 .. occupancy limit):
                 more blocks hide latency, fewer make the grid barriers cheaper
  min_chunk      rows per small-triangle / caster work item (8/16/32): finer
                 items balance big triangles over more lanes, coarser ones
                 repeat less row replay

The semantic tile stays 16 px: the reference restarts its interpolants at
every 16-px tile border, so the tile size is part of the arithmetic that the
bit-exact outputs depend on; only the scheduling granularity is tuned.

The winner is cached per GPU and workload signature in a JSON file
($AXR_TUNING_CACHE, default ~/.cache/axr_tuning.json).
"""
from __future__ import annotations

import json
import os
import time

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "axr_tuning.json")
BLOCKS = (1, 2, 3, 4)
CHUNKS = (8, 16, 32)
PERSISTENT, PHASED = 0, 1


def _cache_path():
    return os.environ.get("AXR_TUNING_CACHE", DEFAULT_CACHE)


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return {}


def signature(batch, ntris):
    views = ",".join(f"{d.kind}:{d.w}x{d.h}" for d in batch.descs)
    return f"{ntris}|{views}"


def _time_renders(batch, flags, aidx, cast, reps):
    import torch
    stream = torch.cuda.ExternalStream(batch.draw.stream_ptr())
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    batch.render(flags, aidx, cast)
    batch.draw.sync()
    a.record(stream)
    for _ in range(reps):
        batch.render(flags, aidx, cast)
    b.record(stream)
    batch.draw.sync()
    return a.elapsed_time(b) / reps


def tune(batch, flags, aidx=None, cast=None, ntris=0, reps=5, gpu="", use_cache=True, log=None):
    """Sweeps the knobs, applies and returns the fastest {mode, blocks_per_sm, min_chunk, ms}."""
    path = _cache_path()
    key = f"{gpu}|{signature(batch, ntris)}"
    cache = _load(path) if use_cache else {}
    if key in cache and "mode" in cache[key]:
        best = cache[key]
        batch.set_mode(best["mode"])
        batch.set_tuning(best["blocks_per_sm"], best["min_chunk"])
        return dict(best, cached=True)
    results = []
    points = [(PERSISTENT, b, c) for b in BLOCKS for c in CHUNKS] + [(PHASED, BLOCKS[-1], c) for c in CHUNKS]
    for mode, bps, ch in points:
        try:
            batch.set_mode(mode)
            batch.set_tuning(bps, ch)
        except Exception:
            continue              # more blocks per SM than the compiled kernel can keep resident
        ms = _time_renders(batch, flags, aidx, cast, reps)
        results.append({"mode": mode, "blocks_per_sm": bps, "min_chunk": ch, "ms": ms})
        if log:
            log(f"autotune mode={'phased' if mode else 'persistent'} blocks/SM={bps} chunk={ch}: {ms:.3f} ms")
    best = min(results, key=lambda r: r["ms"])
    batch.set_mode(best["mode"])
    batch.set_tuning(best["blocks_per_sm"], best["min_chunk"])
    if use_cache:
        cache = _load(path)
        cache[key] = dict(best, when=time.strftime("%Y-%m-%dT%H:%M:%S"))
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            with open(path, "w") as f:
                json.dump(cache, f, indent=1)
        except OSError:
            pass
    return dict(best, cached=False, sweep=results)
