"""Generates the deep-octree golden fixtures from the reference's own code
(oracle/_ref, compiled unmodified by `make -C oracle ref`).  Run in a machine
that has the reference sources:

    python tests/golden/make_golden_deep.py [c1|c4|all]

The benchmark configurations build deeper octrees than config 0 (depth 3):
  * c1: the 512^3 cumulus (workloads.cumulus_recipe), octree depth 6,
        sigma_t 60, albedo 0.999, 64 scattering events;
  * c4: four puffs of the large sparse scene (workloads.slab_recipe puffs 15,
        23, 6, 12, chosen far apart so that the root box spans the slab) on
        its 2048^3 grid, octree depth 8, sigma_t 100, albedo 0.99, 128 events.
Each octree is built by the C restatement of the scene build (oracle/port,
which the product builder reproduces bit for bit).  Fixtures per config:
  ref_<c>_leaf_sequences.npz
      the octree's node records (no bricks: traversal reads nodes only), the
      SHA-256 of its brick pool, and the leaf sequences with (tr0, tr1) of
      RAYS rays from the reference's step traverser (OctreeStepTraverser,
      src/KernelOctree.cpp:230-349), ragged: seq_* concatenated, offsets in
      `start` (the full traverser, :128-220, gives the same lists: checked
      here before writing);
  ref_<c>_crop.npz
      RUNS independent reference renders (RenderKernel::Render,
      src/kernel.cpp:536-567) of a 32x32 crop at SPP samples: per run the
      sums of each buffer and channel over the crop and over its 4x4 blocks
      of 8x8 pixels, plus the mean image over the runs.
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "droplet-render_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle import Port, Reference  # noqa: E402
from deep_configs import CONFIGS, block_stats, build_field, crop_cfg, ray_set  # noqa: E402

RUNS, SPP = 16, 256


def make(name: str, ref: Reference, port: Port):
    c = CONFIGS[name]
    t = time.time()
    org, vals, rec = build_field(name, device="cpu")
    nodes, bricks, mlevel = port.build_octree(org, vals, rec.voxel_size, 12)
    print(f"{name}: {len(org)} blocks, {len(nodes)} nodes, {len(bricks)} leaves, depth {mlevel} "
          f"({time.time() - t:.1f}s)", flush=True)
    assert mlevel == c["depth"], mlevel
    rs = ref.scene(nodes, bricks)
    ro, rd = ray_set(nodes, c["rays"], seed=c["ray_seed"])
    seqs, start = [], [0]
    for i in range(len(ro)):
        s = rs.leaf_sequence(ro[i], rd[i], full=False, maxn=4096)
        f = rs.leaf_sequence(ro[i], rd[i], full=True, maxn=4096)
        for a, b in zip(s, f):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), i
        seqs.append(s)
        start.append(start[-1] + len(s[0]))
    counts = np.diff(start)
    print(f"{name}: {len(ro)} rays, {counts.sum()} leaves, max {counts.max()} per ray", flush=True)
    np.savez_compressed(
        os.path.join(HERE, f"ref_{name}_leaf_sequences.npz"),
        nodes=nodes.view(np.uint8), mlevel=mlevel, n_leaves=len(bricks),
        bricks_sha256=np.frombuffer(hashlib.sha256(bricks.tobytes()).digest(), np.uint8),
        ro=ro, rd=rd, start=np.asarray(start, np.int64),
        seq_node=np.concatenate([s[0] for s in seqs]).astype(np.uint32),
        seq_tr0=np.concatenate([s[1] for s in seqs]).astype(np.float32),
        seq_tr1=np.concatenate([s[2] for s in seqs]).astype(np.float32))

    pdf, cdf = ref.mie_tables()
    sd = crop_cfg(name, pdf, cdf, None, None)[0]["sun_dir"]
    cfgs, rads = ref.sky_state(3.0, 0.3, ref.solar_elevation(sd))  # the harness cooks the same state itself
    cfg, (x0, y0) = crop_cfg(name, pdf, cdf, cfgs, rads)
    ref.set_threads(0)
    t = time.time()
    totals, blocks, acc = [], [], None
    for k in range(RUNS):
        sun, sky = rs.render(cfg, x0, y0, 32, 32, SPP)
        img = np.stack([sun, sky]).astype(np.float64)
        acc = img if acc is None else acc + img
        tot, blk = block_stats(img)
        totals.append(tot)
        blocks.append(blk)
    print(f"{name}: {RUNS} reference renders of 32x32 at {SPP} spp in {time.time() - t:.1f}s", flush=True)
    np.savez_compressed(os.path.join(HERE, f"ref_{name}_crop.npz"), totals=np.asarray(totals),
                        blocks=np.asarray(blocks), mean=(acc / RUNS).astype(np.float32), runs=RUNS, spp=SPP,
                        x0=x0, y0=y0)


def main():
    which = sys.argv[1] if len(sys.argv) > 1 else "all"
    ref, port = Reference(), Port()
    for name in (["c1", "c4"] if which == "all" else [which]):
        make(name, ref, port)


if __name__ == "__main__":
    main()
