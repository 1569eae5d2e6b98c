"""The CPU restatement (oracle/port) pinned against the reference's own code:
the golden vectors it produced (tests/golden, made by make_golden.py from the
unmodified reference sources) and, where the compiled reference is present,
the reference itself."""
import ctypes as C

import numpy as np
import pytest

from conftest import c0_cfg, golden, golden_octree, mie_table


def _params(port, cfg):
    keep = []
    return port.params(cfg, keep), keep


def test_port_builder_matches_golden_octree(port):
    z = golden("c0_octree.npz")
    nodes, bricks, mlevel = port.build_octree(z["block_origin"], z["block_values"], 1.0 / 64, 12)
    g_nodes, g_bricks, g_ml = golden_octree()
    assert mlevel == g_ml == 3
    assert nodes.tobytes() == g_nodes.tobytes()
    assert bricks.tobytes() == g_bricks.tobytes()


def test_last_created_node_is_not_resampled(port):
    """src/scene.cpp:870 resamples nodes [0, index): the last node keeps majorant 0."""
    nodes, bricks, _ = golden_octree()
    last = nodes[-1]
    assert last["volx"][1] != 0xFFFFFFFF
    assert last["qval"][1] == 0.0
    assert not bricks[last["volx"][1]].any()
    others = nodes[:-1][nodes[:-1]["volx"][:, 1] != 0xFFFFFFFF]
    assert (others["qval"][:, 1] >= 0.01).all()


def test_port_leaf_sequences_match_reference_vectors(port):
    nodes, _, _ = golden_octree()
    z = golden("ref_leaf_sequences.npz")
    for i in range(len(z["ro"])):
        n, a, b = port.leaf_sequence(nodes, z["ro"][i], z["rd"][i], maxn=z["nodes"].shape[1])
        k = int(z["count"][i])
        assert len(n) == k
        assert np.array_equal(n, z["nodes"][i, :k])
        assert np.array_equal(a.view(np.uint32), z["tr0"][i, :k].view(np.uint32))
        assert np.array_equal(b.view(np.uint32), z["tr1"][i, :k].view(np.uint32))


def test_port_leaf_sequences_match_reference_live(port, ref):
    nodes, bricks, _ = golden_octree()
    rs = ref.scene(nodes, bricks)
    rng = np.random.default_rng(7)
    for i in range(3000):
        ro = rng.uniform(-1.5, 2.5, 3).astype(np.float32) if i % 3 else rng.uniform(0.1, 0.9, 3).astype(np.float32)
        rd = rng.normal(size=3)
        if i % 50 == 0:
            rd = np.zeros(3)
            rd[i % 3] = 1.0 if i % 2 else -1.0  # axis-parallel rays
        rd = (rd / np.linalg.norm(rd)).astype(np.float32)
        p = port.leaf_sequence(nodes, ro, rd)
        for full in (False, True):
            r = rs.leaf_sequence(ro, rd, full=full)
            assert np.array_equal(p[0], r[0])
            assert np.array_equal(p[1].view(np.uint32), r[1].view(np.uint32))
            assert np.array_equal(p[2].view(np.uint32), r[2].view(np.uint32))


def test_port_point_lookup_is_consistent_with_traversal(port):
    """FP64 point location agrees with the leaf the traversal reports around the point."""
    nodes, _, _ = golden_octree()
    rng = np.random.default_rng(3)
    leaves = np.nonzero(nodes["volx"][:, 1] != 0xFFFFFFFF)[0]
    for leaf in rng.choice(leaves, 64):
        c, e = nodes["ce"][leaf][:3].astype(np.float64), float(nodes["ce"][leaf][3])
        p = c + rng.uniform(-0.9, 0.9, 3) * e
        got, depth = port.point_lookup(nodes, p)
        assert got == leaf and depth == 2


def test_port_sample_voxel_space_matches_reference_vectors(port):
    nodes, bricks, _ = golden_octree()
    z = golden("ref_samplers.npz")
    for i in range(len(z["leaf"])):
        leaf = z["leaf"][i]
        v = port.sample_voxel_space(z["pts"][i], bricks[nodes["volx"][leaf, 1]], nodes["ce"][leaf])
        assert np.float32(v).view(np.uint32) == z["density"][i].view(np.uint32)


def test_port_mie_matches_reference_vectors(port):
    z = golden("ref_samplers.npz")
    P, keep = _params(port, c0_cfg(8, 8))
    out = np.zeros(3, np.float32)
    for i in range(len(z["ct"])):
        port.L.orc_mie_eval_rgb(C.byref(P), float(z["ct"][i]), out.ctypes.data)
        assert np.array_equal(out.view(np.uint32), z["mie_rgb"][i].view(np.uint32))
    d = np.zeros(3, np.float32)
    for i in range(len(z["u1"])):
        port.L.orc_mie_sample(C.byref(P), z["iv"][i].ctypes.data, float(z["u1"][i]), float(z["u2"][i]), d.ctypes.data)
        # sin/cos differ from the reference's SSE approximations by ulps only
        assert np.abs(d - z["mie_dir"][i]).max() < 4e-6
        port.L.orc_sun_sample(C.byref(P), float(z["u1"][i]), float(z["u2"][i]), d.ctypes.data)
        assert np.abs(d - z["sun_dir"][i]).max() < 2e-6


def test_mie_bisection_equals_reference_scan(port):
    """The GPU samples the reference's scan by bisection; both give the same bin."""
    P, keep = _params(port, c0_cfg(8, 8))
    rng = np.random.default_rng(11)
    u = np.concatenate([rng.random(50000), np.linspace(0, 1, 20001)[1:-1]]).astype(np.float32)
    for x in u:
        a = port.L.orc_mie_sample_theta_scan(C.byref(P), float(x))
        b = port.L.orc_mie_sample_theta_bisect(C.byref(P), float(x))
        assert np.float32(a).view(np.uint32) == np.float32(b).view(np.uint32)


def test_reference_mie_sampler_fails_chi_square(ref):
    """Documents the reference sampler's bias (it never draws the last two theta bins)."""
    pdf, cdf = ref.mie_tables()
    rng = np.random.default_rng(5)
    n = 400000
    iv = np.tile(np.array([[0.0, 0.0, 1.0]], np.float32), (n, 1))
    d = ref.mie_sample(iv, rng.random(n).astype(np.float32), rng.random(n).astype(np.float32))
    theta_idx = np.clip((np.arccos(np.clip(-d[:, 2], -1, 1)) / np.pi * 256).astype(int), 0, 255)
    assert (theta_idx >= 254).sum() == 0
    assert cdf[253, 0] < 0.999  # the last two bins hold probability mass in the table


def test_fp64_optical_depth_matches_riemann(port):
    nodes, bricks, _ = golden_octree()
    S = port.scene(nodes, bricks)
    ro = np.array([0.5, -1.5, 0.45], np.float64)
    rd = np.array([0.05, 1.0, 0.02])
    rd /= np.linalg.norm(rd)
    tau = port.L.orc_optical_depth(C.byref(S), ro.ctypes.data, rd.ctypes.data, 10.0)
    # midpoint rule on a fine grid along the same leaf intervals, in float64
    n, a, b = port.leaf_sequence(nodes, ro.astype(np.float32), rd.astype(np.float32))
    acc = 0.0
    for leaf, t0, t1 in zip(n, a, b):
        if nodes["qval"][leaf, 1] == 0.0:
            continue
        ts = np.linspace(max(t0, 0.0), t1, 20001)
        tm = 0.5 * (ts[1:] + ts[:-1])
        brick = bricks[nodes["volx"][leaf, 1]]
        ce = nodes["ce"][leaf]
        vals = [port.sample_voxel_space((ro + rd * t).astype(np.float32), brick, ce) for t in tm[::50]]
        acc += np.mean(vals) * (t1 - max(t0, 0.0))
    assert tau > 0.01
    assert abs(tau - acc) / tau < 5e-3


def test_port_render_matches_reference_statistically(port, ref):
    """The loop form of SampleVolume (port) has the reference's expectation:
    image sums of 4 independent runs each agree within 4 standard errors."""
    nodes, bricks, _ = golden_octree()
    cfg = c0_cfg(24, 24)
    rs = ref.scene(nodes, bricks)
    ref.set_threads(0)
    P, keep = _params(port, cfg)
    S = port.scene(nodes, bricks)
    spp = 4096
    R = [rs.render(cfg, 0, 0, 24, 24, spp) for _ in range(4)]
    Q = [port.render_tile(S, P, 0, 0, 24, 24, spp, seed=1000 + k)[:2] for k in range(4)]
    for bi in range(2):
        for ch in range(4):
            r = np.array([x[bi][..., ch].sum() / spp for x in R])
            q = np.array([x[bi][..., ch].sum() / spp for x in Q])
            assert np.isfinite(r).all()
            se = np.sqrt(r.var(ddof=1) / 4 + q.var(ddof=1) / 4) + 1e-12 * abs(r.mean())
            assert abs(r.mean() - q.mean()) < 4.0 * se + 1e-7, (bi, ch, r.mean(), q.mean(), se)
