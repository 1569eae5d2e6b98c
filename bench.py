"""Benchmark of the droplet_b200 hot path: path-vertices/s of the plain renderer.

Workload (one step = one frame): the single large cumulus, a 512^3 field made of
the config-0 puff plus three offset copies, sigma_t = 60, albedo 0.999, Mie
phase table, sun at 30 degrees plus Hosek sky (T = 3, ground albedo 0.3),
1920x1080, 64 spp, at most 64 scattering events, binary32.  Inputs are seeded
synthetic data (workloads.cumulus_recipe); no dataset is involved.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun each rank renders its own frame with its own sample streams
(independent units, no collective): scaling is weak, value = all ranks'
vertices / the slowest rank's time.

The --impl reference arm times the reference renderer's own CPU code
(oracle/_ref: src/kernel.cpp etc. compiled unmodified) on the host cores over a
bounded crop of the same frame; its vertex count comes from the CPU
restatement (same estimator, counted), as the reference code is not
instrumented.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "droplet-render_b200"))
sys.path.insert(0, ROOT)

from droplet_b200 import camera as cam  # noqa: E402
from droplet_b200 import workloads as W  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")
W_IMG, H_IMG, SPP = 1920, 1080, 64
METRIC = "path-vertices/s (plain renderer, single large cumulus 512^3, 1920x1080, 64 spp)"
CPU_CROP = 384  # reference / cpu_baseline sample: centre crop at full spp (about 10 s of 16 cores)
TRAVERSALS = {0: "octree stack traversal (local memory)", 1: "leaf-grid cell walk",
              2: "octree stack traversal (shared memory)"}
PHASE_SAMPLER = ("the reference's Mie sampler (src/KernelSampler.cpp:258-273: interpolated scan of the red CDF), "
                 "reproduced for image parity; it fails a chi-square test against its own table (the last two "
                 "theta bins are never drawn); DR_PHASE_MIE_EXACT is the sampler that passes")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def load_inputs():
    z = np.load(os.path.join(GOLDEN, "mie_reference_table.npz"))
    pdf, cdf = np.ascontiguousarray(z["pdf"], np.float32), np.ascontiguousarray(z["cdf"], np.float32)
    with open(os.path.join(GOLDEN, "sky_states.json")) as f:
        st = next(s for s in json.load(f) if s["note"] == "c0/c1 sun")
    return pdf, cdf, np.asarray(st["configs"]), np.asarray(st["radiances"])


def frame_cfg(pdf, cdf, cfgs, rads) -> dict:
    sd = cam.sun_direction(W.SUN["elevation"], W.SUN["azimuth"])
    eye = cam.orbit_eye(W.CENTER, W.CAMERA["distance"], W.CAMERA["azimuth"], W.CAMERA["elevation"])
    viewi, proji = cam.camera_matrices(eye, W.CENTER, W.CAMERA["fov"], W_IMG, H_IMG)
    ss, sa, ev = W.medium("c1")
    return dict(sigma_s=ss, sigma_a=sa, scattevs=ev, sun_dir=sd, sun_color=np.asarray(W.SUN["color"], np.float32),
                sun_angle=W.SUN["angle"], turbidity=W.SKY["turbidity"], ground_albedo=W.SKY["albedo"],
                sky_configs=cfgs, sky_radiances=rads, mie_pdf=pdf, mie_cdf=cdf, viewi=viewi, proji=proji, w=W_IMG,
                h=H_IMG)


def build_scene(builder: str):
    rec = W.cumulus_recipe(512)
    t = time.time()
    org, vals = W.sparse_field_fast(rec)
    log(f"field: {len(org)} blocks in {time.time() - t:.1f}s")
    t = time.time()
    if builder == "product":
        from droplet_b200.scene import build_octree

        oc = build_octree(org, vals, rec.voxel_size, 12)
        nodes, bricks, mlevel = oc.nodes, oc.bricks, oc.mlevel
    else:
        from oracle import Port

        nodes, bricks, mlevel = Port().build_octree(org, vals, rec.voxel_size, 12)
    log(f"octree: {len(nodes)} nodes, {len(bricks)} leaves, depth {mlevel}, {time.time() - t:.1f}s")
    return nodes, bricks, mlevel, float((vals != 0).sum()) / 512 ** 3


def crop_box(n=CPU_CROP):
    return (W_IMG - n) // 2, (H_IMG - n) // 2, n, n


def batched_workload(pdf, cdf):
    """Scenes and per-view settings of the batched workload (workloads.c2_batch)."""
    from droplet_b200.renderer import PhaseTable, RenderSettings
    from droplet_b200.scene import build_octree
    from droplet_b200.sky import SkyState

    with open(os.path.join(GOLDEN, "sky_states_by_degree.json")) as f:
        sky = {s["degree"]: s for s in json.load(f)}
    fields, views = W.c2_batch()
    scenes = []
    for fd in fields:
        rec = W.config0_recipe(fd["n"], fd["seed"])
        org, vals = W.sparse_field_fast(rec)
        scenes.append(build_octree(org, vals, rec.voxel_size, 12))
    settings = []
    for v in views:
        fd, side = fields[v["field"]], v["side"]
        eye = cam.orbit_eye(W.CENTER, W.CAMERA["distance"], v["azimuth"], W.CAMERA["elevation"])
        viewi, proji = cam.camera_matrices(eye, W.CENTER, W.CAMERA["fov"], side, side)
        ss, sa, ev = W.medium_of(fd["sigma_t"], W.C2_ALBEDO, W.C2_SCATTEVS)
        st = sky[v["sun_elevation"]]
        settings.append(RenderSettings(
            sigma_s=ss, sigma_a=sa, scattevs=ev, sun_dir=cam.sun_direction(v["sun_elevation"], W.SUN["azimuth"]),
            sun_color=np.asarray(W.SUN["color"], np.float32), sun_angle=W.SUN["angle"],
            sky=SkyState(np.asarray(st["configs"]), np.asarray(st["radiances"])), phase=PhaseTable(pdf, cdf),
            viewi=viewi, proji=proji, w=side, h=side))
    return fields, views, scenes, settings


PROBE_SIDE, PROBE_SPP = 256, 8  # batch autotuner's probe: centre crops of every view


def measure_batched(r, pdf, cdf, steps: int, warmup: int):
    """The batched workload (8 fields x 64 views, one persistent launch per step
    replayed from a CUDA graph) against the plain single-frame path on the same
    views: one launch per view (device time), and the addon's call pattern,
    64x64 tiles through the blocking host API (wall time)."""
    import torch

    from droplet_b200 import autotune
    from droplet_b200.renderer import Batch, BatchView

    t = time.time()
    fields, views, scenes, settings = batched_workload(pdf, cdf)
    t_build = time.time() - t
    saved = r.get_tuning()
    bviews = [BatchView(v["field"], settings[i], v["spp"], 100 + i) for i, v in enumerate(views)]
    b = Batch(r, scenes, bviews)
    # the autotuner times a probe batch: every view, centre crop of at most
    # 256^2, 8 spp (a probe of 128^2 crops at 4 spp launched so little work that
    # its tails favoured an event batch 5% slower on the full batch)
    probe = []
    for i, v in enumerate(views):
        c = min(v["side"], PROBE_SIDE)
        o = (v["side"] - c) // 2
        probe.append(BatchView(v["field"], settings[i], PROBE_SPP, 100 + i, (o, o, c, c)))
    pb = Batch(r, scenes, probe)
    # the full batch runs most views in kernels of their own: so does the probe
    pb.set_split(1)
    t = time.time()
    best, table = autotune.tune_batch(pb, "c2-probe", use_cache=False)
    pb.close()
    stream = torch.cuda.Stream()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    # final stage on the batch itself: the probe's choice against the frame's
    # tuned shape (the large views' kernels are the frame's kernel), one timed
    # launch each after one warm-up launch
    finalists = [tuple(best)] + ([tuple(saved)] if saved[0] == 0 and tuple(saved) != tuple(best) else [])
    final_ms = []
    for c in finalists:
        b.set_tuning(*c)
        b.launch(stream.cuda_stream)
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            a.record(stream)
            b.launch(stream.cuda_stream)
            e.record(stream)
        e.synchronize()
        final_ms.append(a.elapsed_time(e))
    best = finalists[int(np.argmin(final_ms))]
    t_tune = time.time() - t
    b.set_tuning(*best)

    def time_launches():
        for _ in range(max(1, warmup)):
            b.launch(stream.cuda_stream)
        stream.synchronize()
        r.reset_counters()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        with torch.cuda.stream(stream):
            for k in range(steps):
                flush.fill_(float(k))
                ev[k][0].record(stream)
                b.launch(stream.cuda_stream)
                ev[k][1].record(stream)
        stream.synchronize()
        return [a.elapsed_time(e) for a, e in ev], r.counters()["vertices"] / steps

    # the library's default graph: views of at least 8 paths per lane of the
    # grid in persistent kernels of their own, the rest in one batched kernel
    split, own = b.get_split()
    ms, verts = time_launches()
    n_paths, _ = b.info()
    batched = verts / (np.mean(ms) / 1e3)
    # every view in the one batched kernel
    b.set_split(0)
    ms1, verts1 = time_launches()
    single = verts1 / (np.mean(ms1) / 1e3)
    b.set_split(split)
    # plain, one launch per view (same samples as the batch's first launch)
    r.set_tuning(*best)
    cur, plain_ms, plain_v = -1, 0.0, 0
    side_max = max(v["side"] for v in views)
    sun = torch.empty((side_max, side_max, 4), device="cuda")
    sky = torch.empty_like(sun)
    for i, v in enumerate(views):
        if v["field"] != cur:
            r.upload(scenes[v["field"]])
            cur = v["field"]
        r.set_params(settings[i])
        # one untimed render of the view first, as the batch is launched before its timing
        r.render_tile_async(0, 0, v["side"], v["side"], v["spp"], 100 + i, 0, sun.data_ptr(), sky.data_ptr(),
                            stream.cuda_stream)
        stream.synchronize()
        r.reset_counters()
        flush.fill_(1.0)
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        r.render_tile_async(0, 0, v["side"], v["side"], v["spp"], 100 + i, 0, sun.data_ptr(), sky.data_ptr(),
                            stream.cuda_stream)
        e.record(stream)
        e.synchronize()
        plain_ms += a.elapsed_time(e)
        plain_v += r.counters()["vertices"]
    plain = plain_v / (plain_ms / 1e3)
    # the addon's pattern: 64x64 tiles, one blocking dr_render_tile each (host buffers)
    cur, t_tiles, tiles_v, n_tiles = -1, 0.0, 0, 0
    for i, v in enumerate(views):
        if v["field"] != cur:
            r.upload(scenes[v["field"]])
            cur = v["field"]
        r.set_params(settings[i])
        r.reset_counters()
        torch.cuda.synchronize()
        t = time.perf_counter()
        for y in range(0, v["side"], 64):
            for x in range(0, v["side"], 64):
                r.render_tile(x, y, min(64, v["side"] - x), min(64, v["side"] - y), v["spp"], seed=100 + i,
                              sample_base=0)
                n_tiles += 1
        t_tiles += time.perf_counter() - t
        tiles_v += r.counters()["vertices"]
    tiles = tiles_v / t_tiles
    b.close()
    small = measure_small_views(r, scenes, settings, views, best, stream, flush, steps, warmup)
    r.set_tuning(*saved)
    return {
        "workload": "8 fields (config-0 puffs, seeds 10-17, {64..512}^3, sigma_t U[10,80]) x 8 views "
                    "(side U[128,1024], spp {16,64,256}, sun U[5,80] deg, 500 events), default_rng(2026)",
        "value": batched, "unit": "vertices/s", "ms_per_launch": float(np.mean(ms)), "launch_ms": ms,
        "vertices_per_launch": verts, "path_indices_per_launch": n_paths,
        "split": {"min_paths": "auto: 8 paths per lane of the grid" if split == Batch.SPLIT_AUTO else split,
                  "views_with_own_kernel": own, "of_views": len(views)},
        "single_kernel": {"value": single, "unit": "vertices/s", "ms_per_launch": float(np.mean(ms1)),
                          "launch_ms": ms1},
        "plain_per_view": {"value": plain, "ms": plain_ms, "launches": len(views)},
        "plain_addon_tiles_64": {"value": tiles, "seconds": t_tiles, "calls": n_tiles},
        "speedup_vs_plain_per_view": batched / plain, "speedup_vs_addon_tiles": batched / tiles,
        "single_kernel_speedup_vs_plain_per_view": single / plain,
        "target_20x_vs_plain": "unmet: one persistent launch of a large view already keeps every SM busy, so a "
                               "batch can only win the launch tails, the per-launch list kernels and the small "
                               "views (see small_views and speedup_vs_addon_tiles)",
        "small_views": small,
        "tuning": {"choice": list(best), "seconds": round(t_tune, 2),
                   "probe": f"centre <={PROBE_SIDE}^2 crops, {PROBE_SPP} spp, every view in a kernel of its own",
                   "final_stage_on_batch_ms": [[list(c), round(m, 2)] for c, m in zip(finalists, final_ms)],
                   "top": [[c, round(m, 3)] for c, m in table[:6]]},
        "graph": "memset outputs and queues -> camera leaf lists of every view -> {a plain persistent kernel per "
                 "large view, one batched persistent kernel over the rest} as independent branches -> step counter",
        "build_s": round(t_build, 1),
        "l2": "flushed before each timed launch (256 MB write)",
    }


def measure_small_views(r, scenes, settings, views, tuning, stream, flush, steps: int, warmup: int,
                        max_paths: int = 1 << 21):
    """The batch's small views (at most max_paths paths, side^2 x spp: a few
    per lane of the persistent grid, 148 SMs x 8 blocks x 128 lanes; when fewer
    than 4 are that small, the 8 views with the fewest paths): one batched
    launch of just those views against one plain launch per view, both
    device-timed.  A view that small leaves most lanes idle in the tail of a
    launch of its own."""
    import torch

    from droplet_b200.renderer import Batch, BatchView

    pick = [i for i, v in enumerate(views) if v["side"] ** 2 * v["spp"] <= max_paths]
    rule = f"views of at most {max_paths} paths"
    if len(pick) < 4:
        pick = sorted(range(len(views)), key=lambda i: views[i]["side"] ** 2 * views[i]["spp"])[:8]
        rule = "the 8 views with the fewest paths"
    b = Batch(r, scenes, [BatchView(views[i]["field"], settings[i], views[i]["spp"], 100 + i) for i in pick])
    b.set_tuning(*tuning)
    for _ in range(max(1, warmup)):
        b.launch(stream.cuda_stream)
    stream.synchronize()
    r.reset_counters()
    ms = []
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush.fill_(float(k))
            a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            b.launch(stream.cuda_stream)
            e.record(stream)
            e.synchronize()
            ms.append(a.elapsed_time(e))
    verts = r.counters()["vertices"] / steps
    b.close()
    batched = verts / (np.mean(ms) / 1e3)
    r.set_tuning(*tuning)
    side_max = max(views[i]["side"] for i in pick)
    sun = torch.empty((side_max, side_max, 4), device="cuda")
    sky = torch.empty_like(sun)
    cur, plain_ms, plain_v = -1, 0.0, 0
    for i in pick:
        v = views[i]
        if v["field"] != cur:
            r.upload(scenes[v["field"]])
            cur = v["field"]
        r.set_params(settings[i])
        # one untimed render of the view first, as the batch is launched before its timing
        r.render_tile_async(0, 0, v["side"], v["side"], v["spp"], 100 + i, 0, sun.data_ptr(), sky.data_ptr(),
                            stream.cuda_stream)
        stream.synchronize()
        r.reset_counters()
        flush.fill_(1.0)
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        r.render_tile_async(0, 0, v["side"], v["side"], v["spp"], 100 + i, 0, sun.data_ptr(), sky.data_ptr(),
                            stream.cuda_stream)
        e.record(stream)
        e.synchronize()
        plain_ms += a.elapsed_time(e)
        plain_v += r.counters()["vertices"]
    plain = plain_v / (plain_ms / 1e3)
    return {"rule": rule, "views": len(pick), "paths": int(sum(views[i]["side"] ** 2 * views[i]["spp"] for i in pick)),
            "batched": {"value": batched, "unit": "vertices/s", "ms": float(np.mean(ms))},
            "plain_per_view": {"value": plain, "unit": "vertices/s", "ms": plain_ms},
            "speedup_vs_plain_per_view": batched / plain}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 100 ms by one
    nvidia-smi process in loop mode, kept for the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None
        self.th = threading.Thread(target=self.run, daemon=True)
        self.recording = False

    def run(self):
        try:
            for line in self.proc.stdout:
                if self.recording:
                    self.rows.append([x.strip() for x in line.split(",")])
        except Exception:
            pass

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th.start()
        except Exception:
            self.proc = None
        return self

    def __enter__(self):
        self.recording = True
        return self

    def __exit__(self, *a):
        time.sleep(0.15)
        self.recording = False

    def close(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.proc = None

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def kernel_source_sha16() -> str:
    """Digest of the CUDA sources (droplet-render_b200/csrc): a profile summary
    records the digest of the build it measured, so a stale one is detected."""
    import hashlib

    d = os.path.join(ROOT, "droplet-render_b200", "csrc")
    h = hashlib.sha256()
    for name in sorted(os.listdir(d)):
        if name.endswith((".cu", ".cuh", ".h", ".cpp")):
            with open(os.path.join(d, name), "rb") as f:
                h.update(name.encode() + b"\0" + f.read())
    return h.hexdigest()[:16]


def profile_lines(name: str) -> dict:
    """`key: value` lines of a committed profile summary (profiles/<name>)."""
    out = {}
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            for line in f:
                if ":" in line and not line.startswith(("|", "#", " ", "*")):
                    k, v = line.split(":", 1)
                    out[k.strip()] = v.strip()
    except OSError:
        pass
    return out


def profiled_l2():
    """L2 figures of the render kernel from the committed ncu summary
    (profiles/render_persistent_kernel_c1.md, lines "l2_throughput_pct: X" and
    "lts_hit_rate: X")."""
    p = os.path.join(ROOT, "profiles", "render_persistent_kernel_c1.md")
    out = {}
    try:
        with open(p) as f:
            for line in f:
                for key in ("l2_throughput_pct", "lts_hit_rate", "alu_pipe_pct", "issue_active_pct",
                            "lanes_per_instruction"):
                    if line.startswith(key + ":"):
                        out[key] = float(line.split(":")[1])
    except Exception:
        pass
    return out or None


def profiled_traffic():
    """DRAM bytes of one full-frame render launch (dram__bytes_read.sum +
    dram__bytes_write.sum) from the committed ncu summary
    (profiles/render_persistent_kernel_c1.md, lines "dram_bytes_per_frame: X",
    "frame_tuning: ..." and "source_sha16: ..."), used only when it measured
    this build's sources."""
    kv = profile_lines("render_persistent_kernel_c1.md")
    if "dram_bytes_per_frame" not in kv:
        return None
    return {"bytes": float(kv["dram_bytes_per_frame"]), "source_sha16": kv.get("source_sha16"),
            "tuning": kv.get("frame_tuning"), "current": kv.get("source_sha16") == kernel_source_sha16()}


def cpu_reference_times(nodes, bricks, cfg, threads: int, steps: int = 1, warmup: int = 0):
    """Wall times of the reference renderer (oracle/_ref) on the crop, one
    RenderKernel::Render call of the crop at full spp per step."""
    from oracle import Reference

    ref = Reference()
    ref.set_threads(threads)
    rs = ref.scene(nodes, bricks)
    x0, y0, tw, th = crop_box()
    for _ in range(warmup):
        rs.render(cfg, x0 + tw // 2, y0 + th // 2, 16, 16, SPP)
    times = []
    for _ in range(steps):
        t = time.perf_counter()
        rs.render(cfg, x0, y0, tw, th, SPP)
        times.append(time.perf_counter() - t)
    return times


def cpu_reference_time(nodes, bricks, cfg, threads: int) -> float:
    return cpu_reference_times(nodes, bricks, cfg, threads, steps=1, warmup=1)[0]


def port_vertices(nodes, bricks, cfg, threads: int) -> int:
    """Vertices of the crop counted by the CPU restatement (same estimator)."""
    from oracle import Port

    port = Port()
    keep = []
    P = port.params(cfg, keep)
    S = port.scene(nodes, bricks)
    x0, y0, tw, th = crop_box()
    _, _, cnt = port.render_tile(S, P, x0, y0, tw, th, SPP, seed=99, threads=threads)
    return cnt["vertices"]


def c0_settings(pdf, cdf, cfgs, rads, w: int = 256, h: int = 256):
    """Config 0: the 64^3 puff (sigma_t 20, albedo 0.99, 8 events) seen by the
    standard camera at w x h; returns (render configuration dict, settings)."""
    from droplet_b200.renderer import PhaseTable, RenderSettings
    from droplet_b200.sky import SkyState

    sd = cam.sun_direction(W.SUN["elevation"], W.SUN["azimuth"])
    eye = cam.orbit_eye(W.CENTER, W.CAMERA["distance"], W.CAMERA["azimuth"], W.CAMERA["elevation"])
    viewi, proji = cam.camera_matrices(eye, W.CENTER, W.CAMERA["fov"], w, h)
    ss, sa, ev = W.medium("c0")
    cfg = dict(sigma_s=ss, sigma_a=sa, scattevs=ev, sun_dir=sd, sun_color=np.asarray(W.SUN["color"], np.float32),
               sun_angle=W.SUN["angle"], turbidity=W.SKY["turbidity"], ground_albedo=W.SKY["albedo"],
               sky_configs=cfgs, sky_radiances=rads, mie_pdf=pdf, mie_cdf=cdf, viewi=viewi, proji=proji, w=w, h=h)
    st = RenderSettings(sigma_s=ss, sigma_a=sa, scattevs=ev, sun_dir=sd, sun_color=cfg["sun_color"],
                        sun_angle=W.SUN["angle"], sky=SkyState(cfgs, rads), phase=PhaseTable(pdf, cdf), viewi=viewi,
                        proji=proji, w=w, h=h)
    return cfg, st


def measure_c0(r, pdf, cdf, cfgs, rads, steps: int, warmup: int, cpu: bool, cpu_runs: int = 3):
    """Config 0 timed in full on both sides (the reference's CPU-runnable case):
    the 256x256 frame at 16 spp, 8 events.
      * GPU kernel: CUDA events around each frame on the renderer's stream
        (device buffers; the 256 MB L2 flush before each frame);
      * GPU end to end: dr_render_tile with host buffers (parameters uploaded,
        render, both tiles copied back), host clock;
      * reference CPU: RenderKernel::Render over the whole frame (oracle/_ref,
        all host threads), host clock; its vertex count is the GPU's count on
        the same frame (the same estimator; the reference is not instrumented);
      * seconds to 1% relative RMSE against the reference's converged frame
        (tests/golden/ref_c0_converged_256.npz: two 32768-spp reference
        renders, their noise removed): error e16 of a 16-spp frame, spp
        needed n* = 16 (e16 / 0.01)^2 (MSE falls as 1/spp), checked by a GPU
        render at n* spp; the CPU's n* comes from its own timed frames."""
    import torch

    from droplet_b200 import autotune
    from droplet_b200.scene import build_octree

    z = np.load(os.path.join(GOLDEN, "c0_octree.npz"))
    oc = build_octree(z["block_origin"], z["block_values"], 1.0 / 64, 12)
    cfg, st = c0_settings(pdf, cdf, cfgs, rads)
    spp, w, h = 16, 256, 256
    saved = r.get_tuning()
    r.upload(oc)
    r.set_params(st)
    best, _ = autotune.tune(r, (0, 0, w, h), spp, key="c0", use_cache=False)
    stream = torch.cuda.Stream()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    sun = torch.empty((h, w, 4), device="cuda")
    sky = torch.empty_like(sun)
    with torch.cuda.stream(stream):
        for k in range(warmup):
            r.render_tile_async(0, 0, w, h, spp, 3, k * spp, sun.data_ptr(), sky.data_ptr(), stream.cuda_stream)
    stream.synchronize()
    r.reset_counters()
    ms = []
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush.fill_(float(k))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            r.render_tile_async(0, 0, w, h, spp, 3, (warmup + k) * spp, sun.data_ptr(), sky.data_ptr(),
                                stream.cuda_stream)
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
    cnt = r.counters()
    verts = cnt["vertices"] / steps
    kernel = verts / (np.mean(ms) / 1e3)
    b_v = (64.0 * cnt["node_visits"] + 32.0 * cnt["density_lookups"] + 24.0 * cnt["mie_evals"]) / cnt["vertices"]
    peak, peak_kind = measured_peak()
    frame = (np.zeros((h, w, 4), np.float32), np.zeros((h, w, 4), np.float32))
    r.render_tile(0, 0, w, h, 1, seed=3, sample_base=0, out=frame)
    t0 = time.perf_counter()
    for k in range(steps):
        r.set_params(st)
        r.render_tile(0, 0, w, h, spp, seed=3, sample_base=(warmup + k) * spp, out=frame)
    e2e_s = (time.perf_counter() - t0) / steps

    g = np.load(os.path.join(GOLDEN, "ref_c0_converged_256.npz"))
    R = g["mean"].astype(np.float64)
    ok = g["finite"]
    noise = float(np.asarray(g["noise_mse"]).reshape(-1)[0])
    scale = float((R[ok] ** 2).mean())

    def rel(X):
        m = ok & np.isfinite(X)
        return float(np.sqrt(max(float(((X - R)[m] ** 2).mean()) - noise, 0.0) / scale))

    def gpu_image(n, seed):
        acc = np.zeros((h, w, 3))
        done = 0
        while done < n:
            k = min(4096, n - done)
            a, b = r.render_tile(0, 0, w, h, k, seed=seed, sample_base=done)
            acc += (a + b)[..., :3]
            done += k
        return acc / n

    e16 = float(np.mean([rel(gpu_image(spp, 9100 + i)) for i in range(4)]))
    n_star = int(np.ceil(spp * (e16 / 0.01) ** 2))
    check = rel(gpu_image(n_star, 9200)) if n_star <= 1 << 20 else None
    out = {
        "workload": "c0: 64^3 puff (seed 1), sigma_t 20, albedo 0.99, 8 events, 256x256 at 16 spp, whole frame",
        "same_config": True, "tuning": list(best),
        "gpu": {"value": kernel, "unit": "vertices/s", "ms_per_frame": float(np.mean(ms)), "launch_ms": ms,
                "vertices_per_frame": verts, "paths_per_frame": cnt["paths"] / steps,
                "roofline": {"algorithmic_bytes_per_vertex": b_v, "achieved": b_v * kernel / 1e9, "peak": peak,
                             "unit": "GB/s", "frac": b_v * kernel / 1e9 / peak, "peak_kind": peak_kind,
                             "calibration": "counters of the timed frames"}},
        "gpu_e2e": {"value": verts / e2e_s, "unit": "vertices/s", "ms_per_frame": e2e_s * 1e3,
                    "h2d_bytes_per_step": int(pdf.nbytes / 3 * 4 + cdf.nbytes / 3 + 16 * 4 * 2 + 64),
                    "d2h_bytes_per_step": 2 * w * h * 16},
        "seconds_to_1pct_rmse": {
            "reference_image": "mean of 2 x 32768-spp reference (oracle/_ref) renders, noise removed "
                               "(tests/golden/ref_c0_converged_256.npz)",
            "reference_noise_rel": float(np.sqrt(noise / scale)), "rmse_at_16spp_gpu": e16, "spp_needed": n_star,
            "check_rmse_at_spp_needed": check, "gpu_seconds": n_star / spp * float(np.mean(ms)) / 1e3,
            "gpu_e2e_seconds": n_star / spp * e2e_s},
    }
    if cpu:
        from oracle import Reference

        threads = os.cpu_count() or 1
        ref = Reference()
        ref.set_threads(threads)
        rs = ref.scene(oc.nodes, oc.bricks)
        rs.render(cfg, 96, 96, 16, 16, spp)  # warm-up
        times, errs = [], []
        for _ in range(cpu_runs):
            t = time.perf_counter()
            a, b = rs.render(cfg, 0, 0, w, h, spp)
            times.append(time.perf_counter() - t)
            errs.append(rel((a + b)[..., :3].astype(np.float64) / spp))
        cpu_s = float(np.mean(times))
        cpu_n = int(np.ceil(spp * (float(np.mean(errs)) / 0.01) ** 2))
        out["reference_cpu"] = {"value": verts / cpu_s, "unit": "vertices/s", "cores": threads, "kind": "reference",
                                "s_per_frame": cpu_s, "frame_s": times,
                                "sample": "the whole 256x256 frame at 16 spp per run (RenderKernel::Render)"}
        out["seconds_to_1pct_rmse"].update({"rmse_at_16spp_cpu": float(np.mean(errs)), "spp_needed_cpu": cpu_n,
                                            "cpu_seconds": cpu_n / spp * cpu_s})
        out["gpu_over_reference"] = {"kernel": kernel / (verts / cpu_s), "e2e": (verts / e2e_s) / (verts / cpu_s)}
    r.set_tuning(*saved)
    return out


def c3_views(pdf, cdf, cfgs, rads, n_views: int = 16, side: int = 256):
    """The inverse-rendering workload's views: the config-0 camera and sun at
    n_views evenly spaced azimuths."""
    from droplet_b200.renderer import PhaseTable, RenderSettings
    from droplet_b200.sky import SkyState

    ss, sa, ev = W.medium("c0")
    out = []
    for k in range(n_views):
        eye = cam.orbit_eye(W.CENTER, W.CAMERA["distance"], 360.0 * k / n_views, W.CAMERA["elevation"])
        viewi, proji = cam.camera_matrices(eye, W.CENTER, W.CAMERA["fov"], side, side)
        out.append(RenderSettings(
            sigma_s=ss, sigma_a=sa, scattevs=ev, sun_dir=cam.sun_direction(W.SUN["elevation"], W.SUN["azimuth"]),
            sun_color=np.asarray(W.SUN["color"], np.float32), sun_angle=W.SUN["angle"], sky=SkyState(cfgs, rads),
            phase=PhaseTable(pdf, cdf), viewi=viewi, proji=proji, w=side, h=side, finite_paths=True))
    return out


def measure_adjoint(r, pdf, cdf, cfgs, rads, steps: int = 3, warmup: int = 3, fd_groups: int = 8,
                    fd_spp: int = 32, fd_eps: float = 1e-3):
    """Inverse rendering (config 3): target = the config-0 puff at 128^3, seed 5,
    16 views of 256^2 at 256 spp; parameters = the brick samples of a uniform
    0.3 grid (128^3) and the albedo; L2 image loss; 32 spp per gradient step.
    Times the forward (render of the 16 views) and the adjoint (backward) with
    CUDA events; checks the gradient against central finite differences with
    common random numbers (eps 1e-3, majorants held fixed) on 256 random
    voxels (default_rng(5)): per seed group, the directional derivative along
    random signs on those voxels.  Two difference quotients: of the plain
    render (decisions that flip make it noisy at this eps), and of the
    reweighted replay on the adjoint's own streams (decisions from the base
    bricks weighted by their probability ratios: smooth in eps)."""
    import torch

    from droplet_b200 import adjoint as AD
    from droplet_b200.scene import build_from_dense, build_octree

    t = time.time()
    rec = W.config0_recipe(128, 5)
    org, vals = W.sparse_field_fast(rec)
    target_oc = build_octree(org, vals, rec.voxel_size, 12)
    guess_oc = build_from_dense(np.full((128, 128, 128), 0.3, np.float32), 1.0 / 128, 12)
    views = c3_views(pdf, cdf, cfgs, rads)
    saved = r.get_tuning()
    r.upload(target_oc)
    with torch.no_grad():
        tb = torch.tensor(target_oc.bricks, device="cuda")
        tsun, tsky = AD.render(tb, torch.tensor(0.99, device="cuda"), r,
                               [AD.DiffView(v, 256, 500 + k) for k, v in enumerate(views)])
        target = (tsun + tsky)[..., :3].clone()
    r.upload(guess_oc)
    b = torch.tensor(guess_oc.bricks, device="cuda", requires_grad=True)
    alb = torch.tensor(0.99, device="cuda", requires_grad=True)
    t_setup = time.time() - t
    fw, bw = [], []
    stream = torch.cuda.current_stream()
    for it in range(warmup + steps):
        dv = [AD.DiffView(v, 32, 1000 + 97 * it + k) for k, v in enumerate(views)]
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        sun, sky = AD.render(b, alb, r, dv, majorant_scale=1.05)
        loss = (((sun + sky)[..., :3] - target) ** 2).sum()
        e1.record(stream)
        b.grad = None
        alb.grad = None
        loss.backward()
        e2.record(stream)
        e2.synchronize()
        if it >= warmup:
            fw.append(e0.elapsed_time(e1))
            bw.append(e1.elapsed_time(e2))
    grad = b.grad.detach().clone()
    galb = float(alb.grad)
    # finite differences with common random numbers (eps 1e-3) on 256 voxels
    nl = guess_oc.n_leaves
    rng = np.random.default_rng(5)
    pick = torch.as_tensor(rng.choice(nl * 512, 256, replace=False), device="cuda")
    signs = torch.as_tensor(rng.choice([-1.0, 1.0], 256).astype(np.float32), device="cuda")
    u = torch.zeros(nl * 512, device="cuda")
    u[pick] = signs
    u = u.reshape(nl, 512)
    eps = fd_eps
    base = b.detach().clone()
    r.set_bricks_dev(base.data_ptr(), nl, 1.05)  # majorants with headroom, then held fixed
    img = torch.empty((256, 256, 4), device="cuda")
    img2 = torch.empty_like(img)

    def loss_at(bricks, albedo, seed):
        r.set_bricks_dev(bricks.data_ptr(), nl, 0.0)
        tot = 0.0
        for k, v in enumerate(views):
            r.set_params(AD._with_albedo(v, albedo))
            r.render_tile_async(0, 0, 256, 256, fd_spp, seed + k, 0, img.data_ptr(), img2.data_ptr())
            r.synchronize()
            x = (img.double() + img2.double())[..., :3] / fd_spp
            tot += float((delta[k].double() * x).sum())
        return tot

    def adjoint_at(albedo, seed):
        r.set_bricks_dev(base.data_ptr(), nl, 0.0)
        g = torch.zeros_like(base)
        ga = torch.zeros(1, dtype=torch.float64, device="cuda")
        for k, v in enumerate(views):
            r.set_params(AD._with_albedo(v, albedo))
            d4 = torch.zeros((256, 256, 4), device="cuda")
            d4[..., :3] = delta[k] / fd_spp
            r.adjoint_tile_async(0, 0, 256, 256, fd_spp, seed + k, 0, d4.data_ptr(), d4.data_ptr(), g.data_ptr(),
                                 ga.data_ptr())
            r.synchronize()
        return g, float(ga.item())

    def reweighted_at(pert, seed):
        # decisions from the uploaded base bricks, each weighted by its
        # probability ratio under pert: smooth in the perturbation
        r.set_bricks_dev(base.data_ptr(), nl, 0.0)
        tot = torch.zeros(1, dtype=torch.float64, device="cuda")
        for k, v in enumerate(views):
            r.set_params(AD._with_albedo(v, a0))
            d4 = torch.zeros((256, 256, 4), device="cuda")
            d4[..., :3] = delta[k] / fd_spp
            r.reweighted_loss_async(0, 0, 256, 256, fd_spp, seed + k, 0, d4.data_ptr(), d4.data_ptr(),
                                    pert.data_ptr(), tot.data_ptr())
            r.synchronize()
        return float(tot.item())

    # linearised loss: delta = dL/dI at the base point, so both estimators
    # target the same derivative of the expected image
    a0 = 0.99
    with torch.no_grad():
        dv = [AD.DiffView(v, fd_spp, 50000 + k) for k, v in enumerate(views)]
        sun, sky = AD.render(base, torch.tensor(a0, device="cuda"), r, dv, majorant_scale=0.0)
        delta = 2 * ((sun + sky)[..., :3] - target)
    fd, ad, fa, aa, fr = [], [], [], [], []
    pert_p = (base + eps * u).contiguous()
    pert_m = (base - eps * u).contiguous()
    t = time.time()
    # the one-thread-per-path kernel sums each pixel's 32-sample groups in a
    # fixed order: the two renders of a difference share their rounding
    r.set_tuning(1, 0, 0, 0, 0)
    ea = 1e-3
    for gi in range(fd_groups):
        seed = 70000 + 1000 * gi
        fd.append((loss_at(base + eps * u, a0, seed) - loss_at(base - eps * u, a0, seed)) / (2 * eps))
        fa.append((loss_at(base, a0 + ea, seed) - loss_at(base, a0 - ea, seed)) / (2 * ea))
        fr.append((reweighted_at(pert_p, seed) - reweighted_at(pert_m, seed)) / (2 * eps))
        g, ga = adjoint_at(a0, seed)
        ad.append(float((g * u).sum()))
        aa.append(ga)
    fd, ad, fa, aa, fr = np.array(fd), np.array(ad), np.array(fa), np.array(aa), np.array(fr)
    diff = fd - ad
    r.set_tuning(*saved)
    return {
        "workload": "config-0 puff 128^3 seed 5 target, 16 views 256^2 (target 256 spp), uniform 0.3 guess "
                    f"({guess_oc.n_leaves} leaves x 512 samples), L2 loss, 32 spp per gradient step",
        "forward_ms": float(np.mean(fw)), "adjoint_ms": float(np.mean(bw)),
        "adjoint_over_forward": float(np.mean(bw) / np.mean(fw)),
        "grad_norm": float(grad.norm()), "grad_albedo": galb,
        "fd_check": {"eps": eps, "voxels": 256, "groups": fd_groups, "spp_per_view": fd_spp,
                     "raw_crn_status": "uninformative: at eps 1e-3 the raw common-random-number difference "
                                       "quotient counts flipped real/null decisions, each an O(1) jump, so its "
                                       "standard error exceeds the signal (se_of_diff below)",
                     "independent_checks": [
                         "FP64 single-scatter sun image by quadrature, its exact gradient against the GPU adjoint: "
                         "2% per voxel + 4 SE and 1% in projection on the 256 largest-gradient voxels holding >= 1% "
                         "of their leaf majorant, 5% in projection on the 256 largest of all (near-empty voxels give "
                         "heavy-tailed estimates) (tests/test_gpu_adjoint_fp64.py; the quadrature against the "
                         "estimator and its own central differences in tests/test_single_scatter_fp64.py)",
                         "FP64 transmittance gradient (quadrature) against the GPU transmittance adjoint "
                         "(tests/test_gpu_adjoint.py::test_transmittance_adjoint_equals_restatement_and_fp64)"],
                     "reweighted_note": "the reweighted replay shares the adjoint's likelihood-ratio weights: it "
                                        "checks the adjoint's bookkeeping, not its estimator",
                     "directional_fd": fd.tolist(), "directional_adjoint": ad.tolist(),
                     "mean_fd": float(fd.mean()), "mean_adjoint": float(ad.mean()),
                     "rel_diff_of_means": float(abs(fd.mean() - ad.mean()) / max(abs(ad.mean()), 1e-30)),
                     "se_of_diff": float(diff.std(ddof=1) / np.sqrt(len(diff))),
                     "reweighted": {"eps": eps, "fd": fr.tolist(), "adjoint": ad.tolist(),
                                    "max_rel_diff": float(np.max(np.abs(fr - ad) / np.maximum(np.abs(ad), 1e-30))),
                                    "rel_diff_of_means": float(abs(fr.mean() - ad.mean())
                                                               / max(abs(ad.mean()), 1e-30))},
                     "albedo": {"eps": ea, "fd": fa.tolist(), "adjoint": aa.tolist(),
                                "max_rel_diff": float(np.max(np.abs(fa - aa) / np.maximum(np.abs(fa), 1e-30)))},
                     "seconds": round(time.time() - t, 1)},
        "setup_s": round(t_setup, 1),
    }


def build_large(pdf, cdf, cfgs, rads):
    """The config-4 scene and a settings(w, h) factory for its camera:
    (octree, settings, non-zero voxels, field seconds, build seconds, blocks)."""
    from droplet_b200.renderer import PhaseTable, RenderSettings
    from droplet_b200.scene import build_octree
    from droplet_b200.sky import SkyState

    t = time.time()
    rec = W.slab_recipe(2048)
    org, vals = W.sparse_field_puffwise(rec)
    nonzero = int((vals != 0).sum())
    t_field = time.time() - t
    t = time.time()
    oc = build_octree(org, vals, rec.voxel_size, 12)
    t_build = time.time() - t
    n_blocks = int(len(org))
    del vals
    ss, sa, ev = W.medium("c4")

    def settings(w, h):
        eye = cam.orbit_eye(W.CENTER, W.CAMERA["distance"], W.CAMERA["azimuth"], 25.0)
        viewi, proji = cam.camera_matrices(eye, W.CENTER, W.CAMERA["fov"], w, h)
        return RenderSettings(sigma_s=ss, sigma_a=sa, scattevs=ev,
                              sun_dir=cam.sun_direction(W.SUN["elevation"], W.SUN["azimuth"]),
                              sun_color=np.asarray(W.SUN["color"], np.float32), sun_angle=W.SUN["angle"],
                              sky=SkyState(cfgs, rads), phase=PhaseTable(pdf, cdf), viewi=viewi, proji=proji, w=w,
                              h=h)

    return oc, settings, nonzero, t_field, t_build, n_blocks


def profile_large(crop: int, launches: int = 3, spp: int = 256):
    """Capture case for ncu: the config-4 scene, an crop x crop centre crop of
    its 3840x2160 frame at 256 spp, the launch shape the bench renders the full
    frame with (the shared-memory stack traversal, [0, 8, 24, 2, 0, 3, 2]),
    `launches` launches; prints one line of counters."""
    import torch

    from droplet_b200.renderer import Renderer

    pdf, cdf, cfgs, rads = load_inputs()
    oc, settings, _, _, _, _ = build_large(pdf, cdf, cfgs, rads)
    r = Renderer(0)
    r.upload(oc)
    r.set_params(settings(3840, 2160))
    r.set_tuning(0, 8, 24, 2, 0, 3, 2)
    x0, y0 = (3840 - crop) // 2, (2160 - crop) // 2
    sun = torch.empty((crop, crop, 4), device="cuda")
    sky = torch.empty_like(sun)
    r.reset_counters()
    for k in range(launches):
        r.render_tile_async(x0, y0, crop, crop, spp, 11, k * spp, sun.data_ptr(), sky.data_ptr())
    torch.cuda.synchronize()
    cnt = r.counters()
    print(json.dumps({"profile_large": {"crop": crop, "spp": spp, "launches": launches, "counters": cnt,
                                        "bricks_mb": oc.bricks.nbytes / 1e6}}))
    r.close()


def large_cpu_reference(r, oc, settings_big, crop: int = 64, spp: int = 256):
    """The reference renderer (oracle/_ref, all host threads) on a crop x crop
    block of the large scene's 3840x2160 frame at full spp, centred on puff 15
    (the medium, not the empty sky); its vertex count is the GPU renderer's on
    the same block (the same estimator: the reference is not instrumented)."""
    from oracle import Reference

    threads = os.cpu_count() or 1
    p = np.asarray(W.slab_recipe(2048).puffs[15].center, np.float64)
    vi, pj = settings_big.viewi, settings_big.proji
    ys, xs = np.mgrid[0:2160:8, 0:3840:8]
    ro, rd, _ = cam.camera_rays(vi, pj, 3840, 2160, xs.ravel(), ys.ravel())
    v = p - ro.astype(np.float64)
    d = rd.astype(np.float64)
    k = int(np.argmin(np.linalg.norm(v - (v * d).sum(1, keepdims=True) * d, axis=1)))
    x0, y0 = (int(xs.ravel()[k]) - crop // 2) & ~1, (int(ys.ravel()[k]) - crop // 2) & ~1
    ss, sa, ev = W.medium("c4")
    cfg = dict(sigma_s=ss, sigma_a=sa, scattevs=ev, sun_dir=settings_big.sun_dir, sun_color=settings_big.sun_color,
               sun_angle=settings_big.sun_angle, turbidity=W.SKY["turbidity"], ground_albedo=W.SKY["albedo"],
               viewi=vi, proji=pj, w=3840, h=2160)
    ref = Reference()
    ref.set_threads(threads)
    rs = ref.scene(oc.nodes, oc.bricks)
    t = time.perf_counter()
    rs.render(cfg, x0, y0, crop, crop, spp)
    dt = time.perf_counter() - t
    saved = r.get_tuning()
    r.upload(oc)  # the scene and frame may have changed since (the adjoint step sets its own)
    r.set_params(settings_big)
    r.set_tuning()
    r.reset_counters()
    r.render_tile(x0, y0, crop, crop, spp, seed=11, sample_base=0)
    verts = r.counters()["vertices"]
    r.set_tuning(*saved)
    return {"value": verts / dt, "unit": "vertices/s", "cores": threads, "kind": "reference", "seconds": dt,
            "sample": f"{crop}x{crop} block at ({x0},{y0}) of the 3840x2160 frame (on puff 15) at {spp} spp; vertex "
                      "count measured by the GPU renderer on the same block"}


def measure_large(r, pdf, cdf, cfgs, rads, steps: int = 2, warmup: int = 1, spp: int = 256, cpu: bool = False):
    """The large sparse scene (config 4): 24 puffs (workloads.slab_recipe) on a
    2048^3 grid, sigma_t = 100, albedo 0.99, 128 scattering events, 3840x2160 at
    256 spp rendered as 4 camera tiles of 1920x1080: plain (one launch per tile)
    and batched (one graph launch of the 4 tiles), both timed with CUDA events;
    then one adjoint step at 512x512 (32 spp, L2 loss against a 128-spp render of
    the scene, starting from its bricks scaled by 0.9)."""
    import torch

    from droplet_b200 import adjoint as AD
    from droplet_b200 import autotune
    from droplet_b200.renderer import Batch, BatchView

    oc, settings, nonzero, t_field, t_build, n_blocks = build_large(pdf, cdf, cfgs, rads)
    saved = r.get_tuning()
    r.upload(oc)
    big = settings(3840, 2160)
    r.set_params(big)
    best, _ = autotune.tune(r, (960, 540, 1920, 1080), 16, key="c4", use_cache=False)
    stream = torch.cuda.Stream()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    sun = torch.empty((1080, 1920, 4), device="cuda")
    sky = torch.empty_like(sun)
    tiles = [(tx * 1920, ty * 1080) for ty in range(2) for tx in range(2)]

    def frame(k):
        for (x0, y0) in tiles:
            r.render_tile_async(x0, y0, 1920, 1080, spp, 11, k * spp, sun.data_ptr(), sky.data_ptr(), stream.cuda_stream)

    for k in range(warmup):
        frame(k)
    stream.synchronize()
    r.reset_counters()
    ms = []
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush.fill_(float(k))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            frame(warmup + k)
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
    cnt = r.counters()
    plain = cnt["vertices"] / (sum(ms) / 1e3)
    # the bricks (184 MB) exceed L2: algorithmic bytes per vertex from the
    # timed frames' own counters (stack traversal: the reference's node visits)
    b_v = (64.0 * cnt["node_visits"] + 32.0 * cnt["density_lookups"] + 24.0 * cnt["mie_evals"]) / cnt["vertices"]
    peak, peak_kind = measured_peak()
    achieved = b_v * plain / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": peak_kind, "algorithmic_bytes_per_vertex": b_v,
                "calibration": "counters of the timed frames, " + TRAVERSALS.get(best[3], f"traversal {best[3]}")
                               + (" (node visits are grid cells)" if best[3] == 1 else "")}
    bt = Batch(r, [oc], [BatchView(0, big, spp, 11, (x0, y0, 1920, 1080)) for (x0, y0) in tiles])
    bt.set_tuning(*best)
    for _ in range(warmup):
        bt.launch(stream.cuda_stream)
    stream.synchronize()
    r.reset_counters()
    bms = []
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush.fill_(float(k))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            bt.launch(stream.cuda_stream)
            b.record(stream)
            b.synchronize()
            bms.append(a.elapsed_time(b))
    bcnt = r.counters()
    bt.close()
    batched = bcnt["vertices"] / (sum(bms) / 1e3)
    # one adjoint step at 512x512
    small = settings(512, 512)
    with torch.no_grad():
        tb = torch.tensor(oc.bricks, device="cuda")
        tsun, tsky = AD.render(tb, torch.tensor(0.99, device="cuda"), r, [AD.DiffView(small, 128, 5)])
        target = (tsun + tsky)[..., :3].clone()
    b = (0.9 * tb).clone().requires_grad_(True)
    alb = torch.tensor(0.99, device="cuda", requires_grad=True)
    times = []
    for it in range(2):
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        cs = torch.cuda.current_stream()
        e0.record(cs)
        s1, k1 = AD.render(b, alb, r, [AD.DiffView(small, 32, 100 + it)])
        loss = (((s1 + k1)[..., :3] - target) ** 2).sum()
        e1.record(cs)
        b.grad = None
        loss.backward()
        e2.record(cs)
        e2.synchronize()
        times.append((e0.elapsed_time(e1), e1.elapsed_time(e2)))
    cpu_ref = None
    if cpu:
        try:
            cpu_ref = large_cpu_reference(r, oc, big)
        except Exception as e:  # the reference oracle needs oracle/_ref
            cpu_ref = {"value": None, "sample": f"unavailable: {e}"}
    r.set_tuning(*saved)
    return {
        "reference_cpu": cpu_ref,
        "workload": "24 puffs (seeds 20-43, radii U[0.02,0.12], default_rng(2044)) in a 1x1x0.3 slab on a 2048^3 grid, "
                    "sigma_t 100, albedo 0.99, 128 events, 3840x2160 at 256 spp as 4 tiles of 1920x1080",
        "nonzero_voxels": nonzero, "occupancy": nonzero / 2048 ** 3, "blocks": n_blocks,
        "nodes": int(oc.n_nodes), "leaves": int(oc.n_leaves), "octree_depth": int(oc.mlevel),
        "bricks_mb": oc.bricks.nbytes / 1e6, "field_s": round(t_field, 1), "build_s": round(t_build, 1),
        "tuning": list(best),
        "plain": {"value": plain, "unit": "vertices/s", "ms_per_frame": float(np.mean(ms)), "launch_ms": ms,
                  "vertices_per_frame": cnt["vertices"] / steps, "paths_per_frame": cnt["paths"] / steps,
                  "roofline": roofline},
        "batched": {"value": batched, "unit": "vertices/s", "ms_per_frame": float(np.mean(bms)), "launch_ms": bms},
        "adjoint_512": {"forward_ms": times[-1][0], "adjoint_ms": times[-1][1],
                        "ratio": times[-1][1] / times[-1][0], "spp": 32,
                        "grad_norm": float(b.grad.norm()), "loss": float(loss.detach())},
        "l2": "flushed before each timed frame (256 MB write)",
    }


def seconds_to_rmse(r, stream, region, ms_per_frame: float, target: float = 0.01, ref_spp: int = 4096,
                    chunk: int = 256):
    """Seconds of plain rendering to reach `target` relative RMSE against the
    converged image.  The converged image is the mean of two independent
    ref_spp renders A and B (fresh seeds); the reference's own noise is removed
    with MSE(A, B) / 4.  A 64-spp frame (the step's workload) gives the error
    at 64 spp; MSE falls as 1/spp, so n* = 64 (rmse_64 / target)^2 spp, and
    a render at n* spp (fresh seed) checks the prediction."""
    import torch

    x0, y0, tw, th = region

    def render(spp, seed):
        out = torch.zeros((th, tw, 4), dtype=torch.float64, device="cuda")
        sun = torch.empty((th, tw, 4), dtype=torch.float32, device="cuda")
        sky = torch.empty_like(sun)
        done = 0
        with torch.cuda.stream(stream):
            while done < spp:
                n = min(chunk, spp - done)
                r.render_tile_async(x0, y0, tw, th, n, seed, done, sun.data_ptr(), sky.data_ptr(), stream.cuda_stream)
                out += (sun + sky).double()
                done += n
        stream.synchronize()
        return (out[..., :3] / spp).reshape(-1)

    t = time.time()
    A, B = render(ref_spp, 7001), render(ref_spp, 7002)
    X64 = render(SPP, 7003)
    # pixels whose sums hold a NaN (the reference estimator's 0/0 cases, e.g. a
    # direction with rd.y == 0 in the sky term) are left out, and counted
    ok = torch.isfinite(A) & torch.isfinite(B) & torch.isfinite(X64)
    R = 0.5 * (A + B)
    noise = float(((A - B)[ok] ** 2).mean()) / 4.0
    scale = float((R[ok] ** 2).mean())

    def rel(X, m):
        return float(np.sqrt(max(float(((X - R)[m] ** 2).mean()) - noise, 0.0) / scale))

    e64 = rel(X64, ok)
    n_star = int(np.ceil(SPP * (e64 / target) ** 2))
    check = None
    if n_star <= 4 * ref_spp:
        Xn = render(n_star, 7004)
        check = rel(Xn, ok & torch.isfinite(Xn))
    return {"target": target, "rmse_at_64spp": e64, "spp_needed": n_star, "check_rmse_at_spp_needed": check,
            "seconds": n_star / SPP * ms_per_frame / 1e3,
            "reference_image": f"mean of 2 x {ref_spp} spp GPU renders, its noise removed (MSE(A,B)/4)",
            "reference_noise_rel": float(np.sqrt(noise / scale)), "wall_s": round(time.time() - t, 1),
            "non_finite_values_excluded": int((~ok).sum())}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    pdf, cdf, cfgs, rads = load_inputs()
    cfg = frame_cfg(pdf, cdf, cfgs, rads)
    nodes, bricks, mlevel, occ = build_scene("oracle")
    threads = os.cpu_count() or 1
    times = cpu_reference_times(nodes, bricks, cfg, threads, steps=max(1, args.steps), warmup=min(args.warmup, 1))
    verts = port_vertices(nodes, bricks, cfg, threads)
    dt = float(np.mean(times))
    value = verts / dt
    x0, y0, tw, th = crop_box()
    sample = f"{tw}x{th} centre crop of the 1920x1080 frame at {SPP} spp per step"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "vertices/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded fBm puffs)",
        "config": {"workload": "c1 single large cumulus 512^3, 1920x1080, 64 spp, 64 events", "crop": sample},
        "cpu_baseline": {"value": value, "unit": "vertices/s", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "vertices/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_b200(args):
    import torch
    import torch.distributed as dist

    from droplet_b200 import ranks
    from droplet_b200.renderer import PhaseTable, Renderer, RenderSettings
    from droplet_b200.scene import Octree
    from droplet_b200.sky import SkyState

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))

    pdf, cdf, cfgs, rads = load_inputs()
    cfg = frame_cfg(pdf, cdf, cfgs, rads)
    nodes, bricks, mlevel, occ = build_scene("product")
    settings = RenderSettings(sigma_s=cfg["sigma_s"], sigma_a=cfg["sigma_a"], scattevs=cfg["scattevs"],
                              sun_dir=cfg["sun_dir"], sun_color=cfg["sun_color"], sun_angle=cfg["sun_angle"],
                              sky=SkyState(cfgs, rads), phase=PhaseTable(pdf, cdf), viewi=cfg["viewi"],
                              proji=cfg["proji"], w=W_IMG, h=H_IMG)
    r = Renderer(local)
    r.upload(Octree(nodes, bricks, mlevel))
    r.set_params(settings)
    # a dedicated stream: the kernel and the CUDA events that time it share it
    stream = torch.cuda.Stream()
    if args.crop:
        X0, Y0, TW, TH = crop_box(args.crop)
    else:
        X0, Y0, TW, TH = 0, 0, W_IMG, H_IMG
    sun = torch.empty((TH, TW, 4), dtype=torch.float32, device="cuda")
    sky = torch.empty_like(sun)
    seed = ranks.frame_seed(1000, rank)
    tuning = {"kernel": "persistent", "choice": list(r.get_tuning()), "tuned": False}
    if args.tuning:
        r.set_tuning(*[int(v) for v in args.tuning.split(",")])
        tuning = {"choice": list(r.get_tuning()), "tuned": False, "fixed": True}
    elif not args.no_tune:
        from droplet_b200 import autotune

        t = time.time()
        best, table = autotune.tune(r, (X0, Y0, TW, TH), 8, key=f"c1-{TW}x{TH}", use_cache=False)
        tuning = {"choice": list(best), "tuned": True, "seconds": round(time.time() - t, 2),
                  "candidates_ms_at_8spp": [[c, round(ms, 3)] for c, ms in table]}
        log(f"autotune: best {best} in {time.time() - t:.1f}s")

    def step(k):
        r.render_tile_async(X0, Y0, TW, TH, SPP, seed, k * SPP, sun.data_ptr(), sky.data_ptr(), stream.cuda_stream)

    # L2 (126 MB) is flushed between timed steps by writing a 256 MB buffer
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    with torch.cuda.stream(stream):
        for k in range(args.warmup):
            step(k)
    torch.cuda.synchronize()
    r.reset_counters()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local).start()
    time.sleep(0.3)  # the sampler's first lines
    with clocks, torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.fill_(float(k))
            ev[k][0].record(stream)
            step(args.warmup + k)
            ev[k][1].record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks.close()
    kernel_ms = [a.elapsed_time(b) for a, b in ev]
    t_local = sum(kernel_ms) / 1e3
    cnt = r.counters()
    verts_local = cnt["vertices"]
    t_max, verts = ranks.slowest_and_total(t_local, float(verts_local), device="cuda")
    # our kernels per timed frame: the camera leaf-list kernel and the
    # persistent render kernel (stack traversals of the persistent kernel), else one
    tuned_now = r.get_tuning()
    launches_per_step = 2 if (tuned_now[0] == 0 and tuned_now[3] != 1) else 1
    value = verts / t_max

    # end to end through the public blocking API with host buffers (params upload
    # from host + render + copy of both tile buffers back into the caller's
    # frame buffers, allocated once as a renderer keeps its framebuffer), timed
    # on the host
    frame = (np.zeros((TH, TW, 4), np.float32), np.zeros((TH, TW, 4), np.float32))
    r.render_tile(X0, Y0, TW, TH, 1, seed=seed, sample_base=0, out=frame)  # touches the pages once
    h2d = int(pdf.nbytes / 3 * 4 + cdf.nbytes / 3 + 16 * 4 * 2 + 64)
    e2e_steps = max(1, min(args.steps, 3))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        r.set_params(settings)
        r.render_tile(X0, Y0, TW, TH, SPP, seed=seed, sample_base=(args.warmup + k) * SPP, out=frame)
    t_e2e = (time.perf_counter() - t0)
    t_e2e = ranks.slowest(t_e2e, device="cuda")
    e2e_value = (verts / args.steps) * e2e_steps / t_e2e  # same work per frame
    d2h = 2 * TH * TW * 16

    # Algorithmic bytes per vertex B_v = 64 node visits + 32 density lookups +
    # 24 Mie evaluations, counted on a calibration frame (16 spp, fixed seed)
    # with the octree stack traversal, whose node visits are the reference's.
    saved = r.get_tuning()
    r.set_tuning(0, saved[1], saved[2], 0, saved[4])
    r.reset_counters()
    with torch.cuda.stream(stream):
        r.render_tile_async(X0, Y0, TW, TH, 16, 4242, 0, sun.data_ptr(), sky.data_ptr(), stream.cuda_stream)
    stream.synchronize()
    cal = r.counters()
    r.set_tuning(*saved)
    b_v = (64.0 * cal["node_visits"] + 32.0 * cal["density_lookups"] + 24.0 * cal["mie_evals"]) / cal["vertices"]
    peak, peak_kind = measured_peak()
    bytes_per_step = b_v * cnt["vertices"] / args.steps
    avg_s = t_local / args.steps
    achieved = bytes_per_step / avg_s / 1e9
    traffic = profiled_traffic()
    tuned = ",".join(str(v) for v in r.get_tuning())
    usable = bool(traffic and traffic["current"])
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": peak_kind,
                "traffic": traffic["bytes"] if usable else None,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one full-frame launch "
                                  "(profiles/render_persistent_kernel_c1.md)"
                                  + (f"; captured at tuning {traffic['tuning']}, this run {tuned}" if usable else
                                     "; not used: " + ("no capture" if not traffic else "captured on other sources")),
                "algorithmic_bytes_per_vertex": b_v,
                "calibration": "B_v from a 16-spp frame (seed 4242) with the octree stack traversal"}
    # the scene (23 MB of bricks) is L2-resident: the L2's own throughput as a
    # fraction of its peak and its hit rate, from the committed ncu capture
    l2 = profiled_l2()
    if l2:
        roofline["l2"] = {"frac": l2.get("l2_throughput_pct", float("nan")) / 100.0,
                          "lts_hit_rate": l2.get("lts_hit_rate"),
                          "source": "ncu L2 throughput (% of peak) and lts__t_sector_hit_rate.pct on a 512^2 crop "
                                    "launch (profiles/render_persistent_kernel_c1.md)"}
        # the roof that binds: instruction issue on the ALU pipe (compares,
        # selects and integer work of the octree traversal), same capture
        if "alu_pipe_pct" in l2:
            roofline["issue"] = {"alu_pipe_frac": l2["alu_pipe_pct"] / 100.0,
                                 "issue_active_frac": l2.get("issue_active_pct", float("nan")) / 100.0,
                                 "lanes_per_instruction": l2.get("lanes_per_instruction"),
                                 "source": "ncu sm__inst_executed_pipe_alu, smsp__issue_active and "
                                           "smsp__thread_inst_executed_per_inst_executed on the same 512^2 crop "
                                           "launch (profiles/render_persistent_kernel_c1.md)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            threads = os.cpu_count() or 1
            x0, y0, tw, th = crop_box()
            dt_cpu = cpu_reference_time(nodes, bricks, cfg, threads)
            # the reference is not instrumented: its vertex count is this GPU's
            # count on the same crop (the same estimator in expectation)
            r.reset_counters()
            r.render_tile(x0, y0, tw, th, SPP, seed=seed, sample_base=0)
            v_cpu = r.counters()["vertices"]
            cpu = {"value": v_cpu / dt_cpu, "unit": "vertices/s", "cores": threads, "kind": "reference",
                   "sample": f"{tw}x{th} centre crop of the frame at {SPP} spp, one run of the reference renderer "
                             f"({dt_cpu:.1f}s); vertex count measured by the GPU renderer on the same crop"}
        except Exception as e:  # the reference oracle needs oracle/_ref
            cpu = {"value": None, "unit": "vertices/s", "cores": 0, "kind": "reference", "sample": f"unavailable: {e}"}

    c0 = None
    if rank == 0 and world == 1 and not args.no_c0:
        c0 = measure_c0(r, pdf, cdf, cfgs, rads, steps=max(3, args.steps), warmup=max(3, args.warmup),
                        cpu=not args.no_cpu)
        r.upload(Octree(nodes, bricks, mlevel))
        r.set_params(settings)
        log(f"c0: gpu {c0['gpu']['value'] / 1e9:.3f} G/s ({c0['gpu']['ms_per_frame']:.3f} ms/frame), "
            f"e2e {c0['gpu_e2e']['value'] / 1e9:.3f} G/s, cpu "
            f"{(c0.get('reference_cpu') or {}).get('value', float('nan')) / 1e6:.2f} M/s; s to 1%: gpu "
            f"{c0['seconds_to_1pct_rmse']['gpu_seconds']:.3f}, cpu "
            f"{c0['seconds_to_1pct_rmse'].get('cpu_seconds', float('nan')):.1f}")

    rmse = None
    if rank == 0 and world == 1 and not args.no_rmse:
        rmse = seconds_to_rmse(r, stream, (X0, Y0, TW, TH), t_local / args.steps * 1e3)
        rmse["seconds_e2e"] = rmse["spp_needed"] / SPP * (verts / args.steps) / e2e_value
        if cpu and cpu.get("value"):
            rmse["seconds_cpu_reference"] = rmse["spp_needed"] / SPP * (verts / args.steps) / cpu["value"]
        log(f"s to 1% rmse: {rmse['seconds']:.2f} (spp {rmse['spp_needed']}, check {rmse['check_rmse_at_spp_needed']})")

    adjoint = None
    if rank == 0 and world == 1 and not args.no_adjoint:
        adjoint = measure_adjoint(r, pdf, cdf, cfgs, rads, fd_groups=args.fd_groups, fd_spp=args.fd_spp,
                                  fd_eps=args.fd_eps)
        log(f"adjoint: forward {adjoint['forward_ms']:.1f} ms, adjoint {adjoint['adjoint_ms']:.1f} ms, "
            f"ratio {adjoint['adjoint_over_forward']:.2f}, fd {adjoint['fd_check']['mean_fd']:.4g} "
            f"vs {adjoint['fd_check']['mean_adjoint']:.4g}, reweighted fd max rel diff "
            f"{adjoint['fd_check']['reweighted']['max_rel_diff']:.2e}")

    large = None
    if rank == 0 and world == 1 and not args.no_large:
        large = measure_large(r, pdf, cdf, cfgs, rads, cpu=not args.no_cpu)
        log(f"large: plain {large['plain']['value'] / 1e9:.3f} G/s ({large['plain']['ms_per_frame']:.0f} ms/frame), "
            f"batched {large['batched']['value'] / 1e9:.3f} G/s, adjoint step {large['adjoint_512']['ratio']:.2f}x")

    batched = None
    if rank == 0 and world == 1 and not args.no_batched:
        batched = measure_batched(r, pdf, cdf, steps=2, warmup=1)
        log(f"batched: {batched['value'] / 1e9:.3f} G vertices/s ({batched['split']['views_with_own_kernel']} views "
            f"in kernels of their own), one batched kernel {batched['single_kernel']['value'] / 1e9:.3f}, plain per view "
            f"{batched['plain_per_view']['value'] / 1e9:.3f}, addon tiles {batched['plain_addon_tiles_64']['value'] / 1e9:.3f}")

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "vertices/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded fBm puffs)",
            "config": {"workload": "c1 single large cumulus 512^3 (plain renderer)", "image": [W_IMG, H_IMG],
                       "spp": SPP, "scattevs": 64, "sigma_t": 60.0, "albedo": 0.999, "leaves": int(len(bricks)),
                       "nodes": int(len(nodes)), "octree_depth": int(mlevel), "occupancy": occ,
                       "l2": "flushed between steps (256 MB write)", "region": [X0, Y0, TW, TH],
                       "tuning": tuning, "phase_sampler": PHASE_SAMPLER},
            "e2e": {"value": e2e_value, "unit": "vertices/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": e2e_steps},
            "gpu_launches": args.steps * launches_per_step,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clocks.summary(),
            "seconds_to_1pct_rmse": rmse,
            "c0": c0,
            "batched": batched,
            "adjoint": adjoint,
            "large_sparse": large,
            "counters_per_step": {k: v / args.steps for k, v in cnt.items()},
            "kernel_ms": kernel_ms,
        }
        print(json.dumps(line))
    r.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--crop", type=int, default=0, help="render only an NxN centre crop per step (profiling)")
    ap.add_argument("--no-tune", action="store_true", help="skip the launch-shape autotuner")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-workload measurement")
    ap.add_argument("--no-rmse", action="store_true", help="skip the seconds-to-1%%-RMSE measurement")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the inverse-rendering (adjoint) measurement")
    ap.add_argument("--no-large", action="store_true", help="skip the large sparse scene (config 4)")
    ap.add_argument("--no-c0", action="store_true", help="skip the config-0 whole-frame section")
    ap.add_argument("--profile-large", type=int, default=0,
                    help="profiling case only: an NxN centre crop of the config-4 frame, 3 launches")
    ap.add_argument("--fd-groups", type=int, default=8, help="seed groups of the finite-difference check")
    ap.add_argument("--fd-spp", type=int, default=32, help="spp per view of the finite-difference check")
    ap.add_argument("--fd-eps", type=float, default=1e-3, help="brick-sample step of the finite-difference check")
    ap.add_argument("--tuning", default="", help="fixed launch shape kernel,blocks_per_sm,event_batch,traversal,tile,visits (no tuning)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_large:
        return profile_large(args.profile_large)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
