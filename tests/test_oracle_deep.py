"""The CPU restatement and the product builder against the reference at the
benchmark configurations' octree depths (6 for the cumulus frame, 8 for the
large sparse scene), using fixtures the compiled reference produced
(tests/golden/make_golden_deep.py; scenes and rays in tests/deep_configs.py):
  * leaf sequences with bit-exact (tr0, tr1) of 3,000 rays per octree from the
    reference's traversers (src/KernelOctree.cpp:128-349), including the step
    traverser's pops at stack depths up to 7;
  * the octrees themselves (node records and a digest of the bricks);
  * 32x32 crop renders at 256 spp with each configuration's medium and event
    limit (src/kernel.cpp:128-445): 16 independent runs a side, per-run sums
    over the crop and over 4x4 blocks of 8x8 pixels, Welch z below 4.5
    (crop) and 5 (the 32 block statistics per channel group).
Runs on the CPU; the field synthesis takes about half a minute for the
cumulus."""
import hashlib

import numpy as np
import pytest

from conftest import golden, mie_table, sky_state_c0
from deep_configs import CONFIGS, block_stats, build_field, crop_cfg, max_welch_z
from oracle.oracle import NODE_DTYPE

NAMES = ["c1", "c4"]


def _i(a) -> int:
    """A scalar stored in a fixture (kept as a one-element array)."""
    return int(np.asarray(a).reshape(-1)[0])


def _seqs(name):
    z = golden(f"ref_{name}_leaf_sequences.npz")
    z["nodes"] = z["nodes"].view(NODE_DTYPE).reshape(-1)
    return z


@pytest.fixture(scope="module")
def deep_scenes(port):
    """Octree per configuration built by the restatement from the field recipe."""
    out = {}
    for name in NAMES:
        org, vals, rec = build_field(name, device="cpu")
        nodes, bricks, mlevel = port.build_octree(org, vals, rec.voxel_size, 12)
        out[name] = (nodes, bricks, mlevel, org, vals, rec)
    return out


@pytest.mark.parametrize("name", NAMES)
def test_port_leaf_sequences_match_reference_vectors(port, name):
    z = _seqs(name)
    nodes = z["nodes"]
    assert _i(z["mlevel"]) == CONFIGS[name]["depth"]
    st = z["start"]
    nonempty = 0
    for i in range(len(z["ro"])):
        n, a, b = port.leaf_sequence(nodes, z["ro"][i], z["rd"][i])
        s0, s1 = st[i], st[i + 1]
        assert len(n) == s1 - s0, i
        assert np.array_equal(n, z["seq_node"][s0:s1]), i
        assert np.array_equal(a.view(np.uint32), z["seq_tr0"][s0:s1].view(np.uint32)), i
        assert np.array_equal(b.view(np.uint32), z["seq_tr1"][s0:s1].view(np.uint32)), i
        nonempty += s1 > s0
    assert nonempty > len(z["ro"]) // 2


@pytest.mark.parametrize("name", NAMES)
def test_reference_traversers_reproduce_the_vectors(ref, name):
    """The fixtures are the reference's: its step and full traversers, run here
    on the stored nodes, give them again (traversal reads no bricks)."""
    z = _seqs(name)
    nodes = z["nodes"]
    rs = ref.scene(nodes, np.zeros((_i(z["n_leaves"]), 512), np.float32))
    st = z["start"]
    for i in range(0, len(z["ro"]), 3):
        for full in (False, True):
            n, a, b = rs.leaf_sequence(z["ro"][i], z["rd"][i], full=full)
            assert np.array_equal(n, z["seq_node"][st[i]:st[i + 1]])
            assert np.array_equal(a.view(np.uint32), z["seq_tr0"][st[i]:st[i + 1]].view(np.uint32))
            assert np.array_equal(b.view(np.uint32), z["seq_tr1"][st[i]:st[i + 1]].view(np.uint32))


@pytest.mark.parametrize("name", NAMES)
def test_builders_reproduce_the_reference_scenes(deep_scenes, name):
    """The restatement's build of the recipe is the octree the fixtures were made
    on, and the product builder (dr_build_octree) gives it bit for bit."""
    from droplet_b200.scene import build_octree

    nodes, bricks, mlevel, org, vals, rec = deep_scenes[name]
    z = _seqs(name)
    assert mlevel == _i(z["mlevel"])
    assert nodes.tobytes() == z["nodes"].tobytes()
    assert hashlib.sha256(bricks.tobytes()).digest() == z["bricks_sha256"].tobytes()
    oc = build_octree(org, vals, rec.voxel_size, 12)
    assert oc.nodes.tobytes() == nodes.tobytes() and oc.bricks.tobytes() == bricks.tobytes()


def crop_inputs(name):
    pdf, cdf = mie_table()
    cfgs, rads = sky_state_c0()
    return crop_cfg(name, pdf, cdf, cfgs, rads)


@pytest.mark.parametrize("name", NAMES)
def test_port_crop_matches_reference_statistically(port, deep_scenes, name):
    nodes, bricks, _, _, _, _ = deep_scenes[name]
    g = golden(f"ref_{name}_crop.npz")
    cfg, (x0, y0) = crop_inputs(name)
    assert (x0, y0) == (_i(g["x0"]), _i(g["y0"]))
    keep = []
    P = port.params(cfg, keep)
    S = port.scene(nodes, bricks)
    spp, runs = _i(g["spp"]), _i(g["runs"])
    tot, blk = [], []
    for k in range(runs):
        sun, sky, _ = port.render_tile(S, P, x0, y0, 32, 32, spp, seed=5000 + k)
        t, b = block_stats(np.stack([sun, sky]))
        tot.append(t)
        blk.append(b)
    tot, blk = np.asarray(tot), np.asarray(blk)
    assert g["totals"][:, :, 3].mean() > 0.5 * 1024 * spp  # the crop sees the medium
    assert max_welch_z(g["totals"], tot) < 4.5
    assert max_welch_z(g["blocks"].reshape(runs, -1), blk.reshape(runs, -1)) < 5.0
