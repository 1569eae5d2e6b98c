"""Shadow pass (RenderKernel::Shadow, src/kernel.cpp:569-607) and depth
compositing (KERNEL_DEPTHCOMP, src/kernel.cpp:548-554) on the GPU against the
CPU restatement, which the reference pins statistically (test_oracle_pins)."""
import numpy as np
import pytest

from conftest import c0_cfg, clip_end, depth_texture, golden_octree, settings_from_cfg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def depth_renderer():
    from droplet_b200.renderer import Renderer
    from droplet_b200.scene import Octree

    nodes, bricks, mlevel = golden_octree()
    r = Renderer(0)
    r.upload(Octree(nodes, bricks, mlevel))
    yield r
    r.close()


def _cfg(depthcomp):
    w = h = 64
    cfg = c0_cfg(w, h)
    cfg["depth"] = depth_texture(w, h)
    cfg["depthcomp"] = depthcomp
    return cfg


def test_shadow_tile_equals_restatement(depth_renderer, port):
    """Shadow sums are counts of escaped sun-cone segments (sun(lrd)/colour is 0
    or 1 for a white sun), so the GPU tile equals the restatement's exactly:
    rgb bit for bit, alpha +inf, and the same traced segments and lookups."""
    cfg = _cfg(False)
    depth_renderer.set_params(settings_from_cfg(cfg))
    nodes, bricks, _ = golden_octree()
    keep = []
    P = port.params(cfg, keep)
    S = port.scene(nodes, bricks)
    x0, y0, tw, th, spp = 6, 4, 50, 54, 96
    ref, pcnt = port.shadow_tile(S, P, x0, y0, tw, th, spp, seed=21, sample_base=5)
    depth_renderer.reset_counters()
    got, sky = depth_renderer.render_shadow_tile(x0, y0, tw, th, spp, seed=21, sample_base=5)
    cnt = depth_renderer.counters()
    assert np.array_equal(got[..., :3], ref[..., :3])
    assert np.isposinf(got[..., 3]).all() and np.isposinf(ref[..., 3]).all()
    assert not sky.any()
    for k in ("vertices", "density_lookups", "paths"):
        assert cnt[k] == pcnt[k], (k, cnt[k], pcnt[k])
    # the pass traces something and shadows something
    d = cfg["depth"][y0:y0 + th, x0:x0 + tw]
    active = d < clip_end(cfg["proji"])
    assert pcnt["vertices"] == active.sum() * spp
    assert (got[active][:, 0] < spp).mean() > 0.2


def test_shadow_without_depth_texture_counts_every_sample_lit(depth_renderer, port):
    """No depth texture: depth = FLT_MAX is never before the far plane, nothing
    is traced and each pixel sums the sun-cone test of its samples."""
    cfg = _cfg(False)
    cfg["depth"] = None
    depth_renderer.set_params(settings_from_cfg(cfg))
    nodes, bricks, _ = golden_octree()
    keep = []
    P = port.params(cfg, keep)
    S = port.scene(nodes, bricks)
    ref, _ = port.shadow_tile(S, P, 0, 0, 64, 64, 32, seed=3)
    depth_renderer.reset_counters()
    got, _ = depth_renderer.render_shadow_tile(0, 0, 64, 64, 32, seed=3, sample_base=0)
    assert depth_renderer.counters()["vertices"] == 0
    assert np.array_equal(got[..., :3], ref[..., :3])
    assert (got[..., :3] >= 31).all()


@pytest.mark.parametrize("tuning", [(1, 0, 0, 0), (0, 5, 24, 0), (0, 8, 24, 1)])
def test_depth_compositing_paths_equal_restatement(depth_renderer, port, tuning):
    """KERNEL_DEPTHCOMP: a camera ray passing its depth at a leaf boundary
    escapes (alpha 0); a collision at or beyond the depth counts for alpha but
    does not scatter.  Every kernel family traces the restatement's paths."""
    cfg = _cfg(True)
    depth_renderer.set_params(settings_from_cfg(cfg))
    nodes, bricks, _ = golden_octree()
    keep = []
    P = port.params(cfg, keep)
    S = port.scene(nodes, bricks)
    psun, psky, pcnt = port.render_tile(S, P, 4, 6, 56, 52, 40, seed=9, sample_base=3)
    saved = depth_renderer.get_tuning()
    try:
        depth_renderer.set_tuning(*tuning)
        depth_renderer.reset_counters()
        sun, sky = depth_renderer.render_tile(4, 6, 56, 52, 40, seed=9, sample_base=3)
        cnt = depth_renderer.counters()
    finally:
        depth_renderer.set_tuning(*saved)
    for g, p in ((sun, psun), (sky, psky)):
        assert np.allclose(g, p, rtol=2e-5, atol=1e-6 * np.abs(p).max() + 1e-30)
    for k in ("vertices", "density_lookups", "mie_evals", "paths"):
        assert cnt[k] == pcnt[k], (k, cnt[k], pcnt[k])
    # compositing really cut paths: fewer segments than without it
    cfg2 = _cfg(False)
    P2 = port.params(cfg2, keep)
    _, _, full = port.render_tile(S, P2, 4, 6, 56, 52, 40, seed=9, sample_base=3)
    assert pcnt["vertices"] < full["vertices"]
