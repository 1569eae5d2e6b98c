"""Launch-shape autotuner for the persistent path kernel (single frames and batches).

The persistent kernel has seven knobs (`dr_tuning`):
* the compiled variant, i.e. resident blocks per SM. 4/5/6/8 trade registers for
  occupancy; the smaller register budgets spill a little to L1-resident local memory.
* the event batch: how many lanes of a warp must be waiting on a segment end before
  the warp shades them.
* the traversal: octree descent with a node stack in local memory or in shared
  memory (octrees that keep their leaves at one depth; otherwise the library uses
  the local stack), or the cell walk over the leaf grid (faster where
  leaves are dense along rays, slower through wide empty regions).
* the tile: pixels handed out row-major or square by square (ray coherence).
* the work per loop iteration: how many octree nodes the stack traversal examines
  (0: up to the next leaf) and how many free-flight steps a lane takes before the
  warp moves on; balancing them keeps traversing and tracking lanes busy alike.
* the kernel family (persistent, or one thread per path; single frames only).

`tune` searches in two stages: occupancy x event batch (for both octree stacks)
first, then traversal x tile around the best; each candidate is timed with CUDA events on a dedicated stream.
Results are cached per (GPU name, workload key) in a small JSON file, so a later run
with the same key skips the search.
"""
from __future__ import annotations

import json
import os
import time

from . import _native as N

# occupancy x event batch for both stacks: their best occupancies differ (the
# shared-memory stack frees local memory, so more resident blocks pay)
STAGE1 = [(0, bps, batch, trav, 0, 0, 0) for trav in (0, 2) for bps in (4, 5, 6, 8) for batch in (8, 16, 24)]
PER_PATH = (1, 0, 0, 0, 0, 0, 0)


def stage2(best):
    """Around the best occupancy and event batch: traversal x tile, neighbouring
    event batches, and the work per loop iteration (visits x steps)."""
    k, bps, batch = best[:3]
    out = [(k, bps, batch, trav, tile, 0, 0) for trav in (0, 1, 2) for tile in (0, 8, 16)]
    out += [(k, bps, b2, 0, 0, 0, 0) for b2 in (12, 20, 28, 32) if b2 != batch]
    out += [(k, bps, batch, trav, 0, v, st) for trav in (0, 2) for v in (2, 3, 4, 8) for st in (1, 2, 4)]
    return out


def _cache_path() -> str:
    base = os.environ.get("DROPLET_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "droplet_b200")
    os.makedirs(base, exist_ok=True)
    return os.path.join(base, "tuning.json")


def _load_cache() -> dict:
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except Exception:
        return {}


def _store_cache(d: dict):
    tmp = _cache_path() + f".{os.getpid()}.tmp"
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1)
    os.replace(tmp, _cache_path())


def time_region(renderer, region, spp: int, seed: int, repeats: int, stream, sun, sky) -> float:
    """Milliseconds per render of `region` (x0, y0, w, h) with the current tuning."""
    import torch

    x0, y0, w, h = region
    renderer.render_tile_async(x0, y0, w, h, spp, seed, 0, sun.data_ptr(), sky.data_ptr(), stream.cuda_stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for k in range(repeats):
        renderer.render_tile_async(x0, y0, w, h, spp, seed, (k + 1) * spp, sun.data_ptr(), sky.data_ptr(),
                                   stream.cuda_stream)
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b) / repeats


def time_batch(batch, repeats: int, stream) -> float:
    """Milliseconds per graph launch of a batch with its current tuning."""
    import torch

    batch.launch(stream.cuda_stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(repeats):
        batch.launch(stream.cuda_stream)
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b) / repeats


def search(target, timer, per_path: bool = True):
    """Two-stage search over target.set_tuning(*candidate), then the three fastest
    timed again; returns (best, table)."""
    table = []
    seen = set()

    def run(cands):
        for c in cands:
            if c in seen:
                continue
            seen.add(c)
            target.set_tuning(*c)
            table.append((list(c), timer()))

    run(STAGE1 + ([PER_PATH] if per_path else []))
    best = tuple(min(table, key=lambda r: r[1])[0])
    if best[0] == 0:
        run(stage2(best))
    table.sort(key=lambda r: r[1])
    # the leaders are often within a percent of each other: time the three
    # fastest again, interleaved (clock drift falls on all alike), and keep the
    # lowest median
    top = [tuple(r[0]) for r in table[:3]]
    again = {c: [] for c in top}
    for _ in range(3):
        for c in top:
            target.set_tuning(*c)
            again[c].append(timer())
    medians = {c: sorted(v)[len(v) // 2] for c, v in again.items()}
    best = min(top, key=lambda c: medians[c])
    table = [(list(c), medians[c]) for c in sorted(top, key=lambda c: medians[c])] + \
            [r for r in table if tuple(r[0]) not in again]
    return best, table


def final_stage(target, candidates, timer):
    """Times each distinct candidate shape on the real workload (target.set_tuning,
    then timer()), leaves the fastest set and returns (best, [(shape, ms), ...]).
    A search on a reduced probe (tune_batch) can favour shapes that lose on the
    full workload: its winner and, for example, the frame's tuned shape are
    the usual finalists."""
    shapes, times = [], []
    for c in candidates:
        c = tuple(c)
        if c in shapes:
            continue
        shapes.append(c)
        target.set_tuning(*c)
        times.append(timer())
    if not shapes:
        raise ValueError("final_stage: no candidate")
    i = min(range(len(shapes)), key=lambda k: times[k])
    target.set_tuning(*shapes[i])
    return shapes[i], list(zip(shapes, times))


def _cached(key, target, use_cache):
    import torch

    gpu = torch.cuda.get_device_name(getattr(target, "device", 0))
    ckey = f"{gpu}|{key}"
    cache = _load_cache() if use_cache else {}
    if use_cache and ckey in cache:
        best = tuple(cache[ckey]["best"])
        target.set_tuning(*best)
        return ckey, cache, (best, cache[ckey]["table"])
    return ckey, cache, None


def tune(renderer, region, spp: int, key: str, repeats: int = 2, seed: int = 7, use_cache: bool = True):
    """Picks the fastest launch shape for rendering `region` at `spp` and leaves it
    set on the renderer.  Returns (best, table of (candidate, ms))."""
    import torch

    ckey, cache, hit = _cached(key, renderer, use_cache)
    if hit:
        return hit
    x0, y0, w, h = region
    sun = torch.empty((h, w, 4), dtype=torch.float32, device=f"cuda:{renderer.device}")
    sky = torch.empty_like(sun)
    stream = torch.cuda.Stream(device=renderer.device)
    t0 = time.time()
    best, table = search(renderer, lambda: time_region(renderer, region, spp, seed, repeats, stream, sun, sky))
    renderer.set_tuning(*best)
    if use_cache:
        cache[ckey] = {"best": list(best), "table": table, "seconds": time.time() - t0}
        _store_cache(cache)
    return best, table


def tune_batch(batch, key: str, repeats: int = 2, use_cache: bool = True):
    """tune() for a Batch: times whole graph launches of `batch` (normally a
    reduced probe batch of the same scenes and views) and leaves the best set."""
    import torch

    ckey, cache, hit = _cached(key, batch.renderer, use_cache)
    if hit:
        batch.set_tuning(*hit[0])
        return hit
    stream = torch.cuda.Stream(device=batch.renderer.device)
    t0 = time.time()
    best, table = search(batch, lambda: time_batch(batch, repeats, stream), per_path=False)
    batch.set_tuning(*best)
    if use_cache:
        cache[ckey] = {"best": list(best), "table": table, "seconds": time.time() - t0}
        _store_cache(cache)
    return best, table
