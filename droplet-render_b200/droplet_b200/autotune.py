"""Launch-shape autotuner for the persistent path kernel.

The persistent kernel has four knobs (`dr_tuning`):
* the compiled variant, i.e. resident blocks per SM. 4/5/6/8 trade registers for
  occupancy; the smaller register budgets spill a little to L1-resident local memory.
* the event batch: how many lanes of a warp must be waiting on a segment end before
  the warp shades them.
* the kernel family (persistent, or one thread per path).
* the traversal: octree descent with a node stack, or the cell walk over the leaf
  grid (faster where leaves are dense along rays, slower through wide empty regions).

`tune` renders a representative region with every candidate, times each with CUDA
events on a dedicated stream, and keeps the fastest. Results are cached per (GPU
name, workload key) in a small JSON file, so a later run with the same key skips
the search.
"""
from __future__ import annotations

import json
import os
import time

from . import _native as N

DEFAULT_CANDIDATES = [
    (0, bps, batch, trav)
    for trav in (0, 1)
    for bps in (4, 5, 6, 8)
    for batch in (4, 8, 16, 24)
] + [(1, 0, 0, 0)]


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


def tune(renderer, region, spp: int, key: str, candidates=None, repeats: int = 2, seed: int = 7,
         use_cache: bool = True):
    """Picks the fastest (kernel, blocks_per_sm, event_batch, traversal) for the region and
    leaves it set on the renderer.  Returns (best, table of (candidate, ms))."""
    import torch

    gpu = torch.cuda.get_device_name(renderer.device)
    ckey = f"{gpu}|{key}"
    cache = _load_cache() if use_cache else {}
    if use_cache and ckey in cache:
        best = tuple(cache[ckey]["best"])
        renderer.set_tuning(*best)
        return best, cache[ckey]["table"]
    x0, y0, w, h = region
    sun = torch.empty((h, w, 4), dtype=torch.float32, device=f"cuda:{renderer.device}")
    sky = torch.empty_like(sun)
    stream = torch.cuda.Stream(device=renderer.device)
    saved = renderer.get_tuning()
    table = []
    t0 = time.time()
    for cand in candidates or DEFAULT_CANDIDATES:
        renderer.set_tuning(*cand)
        ms = time_region(renderer, region, spp, seed, repeats, stream, sun, sky)
        table.append((list(cand), ms))
    table.sort(key=lambda r: r[1])
    best = tuple(table[0][0]) if table else saved
    renderer.set_tuning(*best)
    if use_cache:
        cache[ckey] = {"best": list(best), "table": table, "seconds": time.time() - t0}
        _store_cache(cache)
    return best, table
