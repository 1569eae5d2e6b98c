"""The product's host octree builder (dr_build_octree, C ABI) against the
CPU restatement of the reference scene build and the golden config-0 octree.
Host-only: runs without a GPU."""
import numpy as np
import pytest

from conftest import golden, golden_octree
from droplet_b200 import _native as N
from droplet_b200 import workloads as W
from droplet_b200.scene import build_octree


def test_builder_matches_golden_c0():
    z = golden("c0_octree.npz")
    oc = build_octree(z["block_origin"], z["block_values"], 1.0 / 64, 12, threads=3)
    g_nodes, g_bricks, g_ml = golden_octree()
    assert oc.mlevel == g_ml
    assert oc.nodes.tobytes() == g_nodes.tobytes()
    assert oc.bricks.tobytes() == g_bricks.tobytes()


def _random_blocks(rng, nb, span, fill):
    org = rng.choice(span // 8, size=(nb * 3, 3)) * 8
    org = np.unique(org, axis=0)[:nb].astype(np.int32)
    vals = rng.random((len(org), 512)).astype(np.float32)
    vals[rng.random(vals.shape) > fill] = 0.0
    return org, vals


@pytest.mark.parametrize("seed,nb,span,fill,s", [(1, 5, 64, 0.3, 1 / 64), (2, 40, 256, 0.05, 1 / 256),
                                                 (3, 300, 512, 0.5, 1 / 512), (4, 1, 8, 0.01, 0.1),
                                                 (5, 60, 4096, 0.2, 1 / 4096)])
def test_builder_matches_port_on_random_sparse_scenes(port, seed, nb, span, fill, s):
    rng = np.random.default_rng(seed)
    org, vals = _random_blocks(rng, nb, span, fill)
    try:
        p_nodes, p_bricks, p_ml = port.build_octree(org, vals, s, 12)
    except ValueError:
        with pytest.raises(N.DrError):
            build_octree(org, vals, s, 12)
        return
    oc = build_octree(org, vals, s, 12)
    assert oc.mlevel == p_ml
    assert oc.nodes.tobytes() == p_nodes.tobytes()
    assert oc.bricks.tobytes() == p_bricks.tobytes()


def test_builder_c1_recipe_matches_port(port):
    rec = W.cumulus_recipe(128)
    org, vals = W.sparse_field(rec)
    oc = build_octree(org, vals, rec.voxel_size, 12)
    p_nodes, p_bricks, p_ml = port.build_octree(org, vals, rec.voxel_size, 12)
    assert oc.nodes.tobytes() == p_nodes.tobytes() and oc.bricks.tobytes() == p_bricks.tobytes()
    assert oc.mlevel == p_ml


def test_builder_structure_invariants():
    z = golden("c0_octree.npz")
    oc = build_octree(z["block_origin"], z["block_values"], 1.0 / 64, 12)
    nodes = oc.nodes
    leaf = nodes["volx"][:, 1] != N.DR_NONE
    assert not leaf[0]
    assert sorted(nodes["volx"][leaf, 1].tolist()) == list(range(oc.n_leaves))
    # every non-root node is the child of exactly one node, created after its parent (DFS numbering)
    parent = {}
    for i, n in enumerate(nodes):
        for c in n["chn"]:
            if c:
                assert c not in parent and c > i
                parent[int(c)] = i
    assert sorted(parent) == list(range(1, oc.n_nodes))
    assert (oc.bricks >= 0).all() and (oc.bricks <= 1).all()


def test_builder_rejects_bad_input():
    with pytest.raises(N.DrError):
        build_octree(np.zeros((0, 3), np.int32), np.zeros((0, 512), np.float32), 0.1)
    with pytest.raises(N.DrError, match="multiples of 8"):
        build_octree(np.array([[3, 0, 0]], np.int32), np.ones((1, 512), np.float32), 0.1)
    with pytest.raises(N.DrError, match="no active voxels"):
        build_octree(np.array([[0, 0, 0]], np.int32), np.zeros((1, 512), np.float32), 0.1)
    with pytest.raises(N.DrError, match="two octree levels"):
        v = np.zeros((1, 512), np.float32)
        v[0] = 0.5
        build_octree(np.array([[0, 0, 0]], np.int32), v, 0.1)
    with pytest.raises(N.DrError, match="maxdepth"):
        z = golden("c0_octree.npz")
        build_octree(z["block_origin"], z["block_values"], 1.0 / 64, 2)


def test_puffwise_field_equals_blockwise_field():
    """The large scene's generator (each puff on its own blocks, terms summed in
    puff order) gives the values of the block-by-block generator."""
    from droplet_b200 import workloads as W

    rec = W.slab_recipe(96)
    o1, v1 = W.sparse_field(rec)
    o2, v2 = W.sparse_field_puffwise(rec, device="cpu")
    a, b = np.lexsort(o1.T[::-1]), np.lexsort(o2.T[::-1])
    assert len(o1) > 50
    assert np.array_equal(o1[a], o2[b]) and np.array_equal(v1[a], v2[b])
