"""Surface (SDF) leaves (src/kernel.cpp:241-305) in the CPU restatement, pinned
to the compiled reference on a scene whose leaves carry surface bricks (with
and without fog): image sums of 16 independent runs a side agree within 4.5
standard errors, and the opaque sphere covers the pixels it should."""
import numpy as np

from conftest import c0_cfg, golden_octree, sdf_scene

RUNS = 16


def _agree(R, Q, label, z=4.5):
    r, q = np.asarray(R, np.float64), np.asarray(Q, np.float64)
    assert np.isfinite(r).all() and np.isfinite(q).all(), label
    se = np.sqrt(r.var(ddof=1) / len(r) + q.var(ddof=1) / len(q)) + 1e-12 * abs(r.mean())
    assert abs(r.mean() - q.mean()) < z * se + 1e-9, (label, r.mean(), q.mean(), se)


def test_port_sdf_render_matches_reference_statistically(port, ref):
    nodes, bricks, sdf, _ = sdf_scene()
    cfg = c0_cfg(16, 16)
    rs = ref.scene(nodes, bricks, sdf)
    ref.set_threads(0)
    keep = []
    P = port.params(cfg, keep)
    S = port.scene(nodes, bricks, None, sdf)
    spp = 512
    R = [rs.render(cfg, 0, 0, 16, 16, spp) for _ in range(RUNS)]
    Q = [port.render_tile(S, P, 0, 0, 16, 16, spp, seed=3000 + k)[:2] for k in range(RUNS)]
    for bi in range(2):
        for ch in range(4):
            _agree([x[bi][..., ch].sum() / spp for x in R], [x[bi][..., ch].sum() / spp for x in Q], (bi, ch))


def test_sphere_is_opaque(port):
    """Camera rays through the middle of the sphere always collide (alpha 1),
    and the surface darkens what is behind it compared with the fog alone."""
    nodes, bricks, sdf, _ = sdf_scene()
    cfg = c0_cfg(32, 32)
    keep = []
    P = port.params(cfg, keep)
    S = port.scene(nodes, bricks, None, sdf)
    sun, sky, _ = port.render_tile(S, P, 0, 0, 32, 32, 64, seed=4)
    assert (sun[15:17, 14:17, 3] == 64).all()
    fog_nodes, _, _ = golden_octree()
    S0 = port.scene(fog_nodes, bricks)
    sun0, sky0, _ = port.render_tile(S0, P, 0, 0, 32, 32, 64, seed=4)
    assert sun0[15:17, 14:17, 3].sum() < sun[15:17, 14:17, 3].sum()
