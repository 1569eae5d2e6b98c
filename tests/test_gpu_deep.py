"""The GPU path against the reference at the benchmark configurations' octree
depths: the 512^3 cumulus (depth 6; sigma_t 60, albedo 0.999, 64 events) and
four far-apart puffs of the large sparse scene on its 2048^3 grid (depth 8;
sigma_t 100, albedo 0.99, 128 events).  Scenes, rays and crops are those of
tests/deep_configs.py; the fixtures come from the compiled reference
(tests/golden/make_golden_deep.py).

  * the product builder, fed the field synthesised on the GPU, gives the
    octree the fixtures were made on (node records equal, brick digest equal);
  * GPU leaf sequences and (tr0, tr1) of 3,000 rays per octree equal the
    reference traversers' bit for bit (any NaN matches any NaN);
  * GPU path samples of a 16x16 crop equal the CPU restatement's bit for bit
    with every traversal (octree stack in local or shared memory, cell walk,
    one thread per path), the restatement being pinned to the reference at
    these depths by tests/test_oracle_deep.py;
  * 32x32 crops at 256 spp, 16 runs, per traversal: per-run sums over the crop
    and its 4x4 blocks of 8x8 pixels agree with the reference's 16 runs within
    Welch z 4.5 (crop) and 5 (blocks).
"""
import hashlib

import numpy as np
import pytest

from conftest import golden, mie_table, settings_from_cfg, sky_state_c0
from deep_configs import block_stats, build_field, crop_cfg, max_welch_z
from oracle.oracle import NODE_DTYPE

pytestmark = pytest.mark.gpu

NAMES = ["c1", "c4"]
# (kernel, blocks/SM, event batch, traversal, tile, visits, steps)
TUNINGS = [(0, 8, 24, 2, 0, 3, 4), (0, 6, 24, 0, 0, 3, 2), (0, 5, 24, 1, 0, 0, 1), (1, 0, 0, 0, 0, 0, 0)]


def _i(a) -> int:
    return int(np.asarray(a).reshape(-1)[0])


def same_floats(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    nan = np.isnan(a) & np.isnan(b)
    return a.shape == b.shape and bool(((a.view(np.uint32) == b.view(np.uint32)) | nan).all())


@pytest.fixture(scope="module")
def deep():
    """name -> (renderer with the scene uploaded, octree, fixture, cfg, crop origin)."""
    from droplet_b200.renderer import Renderer
    from droplet_b200.scene import build_octree

    pdf, cdf = mie_table()
    cfgs, rads = sky_state_c0()
    out = {}
    for name in NAMES:
        org, vals, rec = build_field(name, device="cuda")
        oc = build_octree(org, vals, rec.voxel_size, 12)
        z = golden(f"ref_{name}_leaf_sequences.npz")
        z["nodes"] = z["nodes"].view(NODE_DTYPE).reshape(-1)
        cfg, xy = crop_cfg(name, pdf, cdf, cfgs, rads)
        r = Renderer(0)
        r.upload(oc)
        r.set_params(settings_from_cfg(cfg))
        out[name] = (r, oc, z, cfg, xy)
    yield out
    for v in out.values():
        v[0].close()


@pytest.mark.parametrize("name", NAMES)
def test_gpu_field_and_builder_give_the_reference_scene(deep, name):
    _, oc, z, _, _ = deep[name]
    assert oc.mlevel == _i(z["mlevel"])
    assert oc.nodes.tobytes() == z["nodes"].tobytes()
    assert hashlib.sha256(oc.bricks.tobytes()).digest() == z["bricks_sha256"].tobytes()


@pytest.mark.parametrize("name", NAMES)
def test_gpu_leaf_sequences_bit_exact_vs_reference(deep, name):
    r, _, z, _, _ = deep[name]
    st = z["start"]
    counts = np.diff(st)
    nodes, a, b, cnt = r.probe_leaf_sequence(z["ro"], z["rd"], int(counts.max()) + 8)
    assert np.array_equal(cnt, counts)
    for i in range(len(cnt)):
        k = int(cnt[i])
        assert np.array_equal(nodes[i, :k], z["seq_node"][st[i]:st[i + 1]]), i
        assert same_floats(a[i, :k], z["seq_tr0"][st[i]:st[i + 1]]), i
        assert same_floats(b[i, :k], z["seq_tr1"][st[i]:st[i + 1]]), i


@pytest.mark.parametrize("name", NAMES)
def test_gpu_paths_equal_restatement_at_depth(deep, port, name):
    r, oc, _, cfg, (x0, y0) = deep[name]
    keep = []
    P = port.params(cfg, keep)
    S = port.scene(oc.nodes, oc.bricks)
    psun, psky, pcnt = port.render_tile(S, P, x0 + 8, y0 + 8, 16, 16, 8, seed=21, sample_base=0)
    assert pcnt["mie_evals"] > 100
    try:
        for tuning in TUNINGS:
            r.set_tuning(*tuning)
            r.reset_counters()
            sun, sky = r.render_tile(x0 + 8, y0 + 8, 16, 16, 8, seed=21, sample_base=0)
            cnt = r.counters()
            for g, p in ((sun, psun), (sky, psky)):
                assert np.allclose(g, p, rtol=2e-5, atol=1e-6 * np.abs(p).max() + 1e-30), tuning
            for k in ("vertices", "density_lookups", "mie_evals", "paths"):
                assert cnt[k] == pcnt[k], (tuning, k)
            if tuning[3] != 1:  # the stack traversals examine the reference's nodes
                assert cnt["node_visits"] == pcnt["node_visits"], tuning
    finally:
        r.set_tuning()


@pytest.mark.parametrize("name", NAMES)
def test_gpu_crop_matches_reference_statistically(deep, name):
    r, _, _, _, (x0, y0) = deep[name]
    g = golden(f"ref_{name}_crop.npz")
    assert (x0, y0) == (_i(g["x0"]), _i(g["y0"]))
    spp, runs = _i(g["spp"]), _i(g["runs"])
    try:
        for tuning in TUNINGS:
            r.set_tuning(*tuning)
            tot, blk = [], []
            for k in range(runs):
                sun, sky = r.render_tile(x0, y0, 32, 32, spp, seed=5000 + k, sample_base=0)
                t, b = block_stats(np.stack([sun, sky]))
                tot.append(t)
                blk.append(b)
            tot, blk = np.asarray(tot), np.asarray(blk)
            assert max_welch_z(g["totals"], tot) < 4.5, tuning
            assert max_welch_z(g["blocks"].reshape(runs, -1), blk.reshape(runs, -1)) < 5.0, tuning
    finally:
        r.set_tuning()
