"""Two performance features of the persistent kernel that must not change any
path: the camera leaf lists (each pixel's camera ray traversed once per launch,
its samples reading the leaf sequence) and the per-warp queue of sky terms
(evaluated 32 at a time).  Against the CPU restatement on the config-0 scene:

  * the default pool, no lists, and a pool too small for most pixels (whose
    samples then traverse) give tiles equal to the restatement's up to the
    order of the per-pixel float sums, with every counter (node visits
    included) exactly equal, through the blocking and the asynchronous call;
  * with the whole-path finiteness check the sky terms are added in place (the
    check needs the path's sum), and the tile still equals the restatement's;
  * a batch renders the same paths with and without lists.
"""
import numpy as np
import pytest

from conftest import c0_cfg, golden_octree, settings_from_cfg
from droplet_b200 import _native as N

pytestmark = pytest.mark.gpu

KEYS = ("paths", "vertices", "node_visits", "density_lookups", "mie_evals")
TILE = (4, 6, 56, 52)


@pytest.fixture(scope="module")
def scene():
    from droplet_b200.renderer import Renderer
    from droplet_b200.scene import Octree

    nodes, bricks, mlevel = golden_octree()
    r = Renderer(0)
    r.upload(Octree(nodes, bricks, mlevel))
    yield r, nodes, bricks, mlevel
    r.close()


def _port_tile(port, cfg, nodes, bricks, spp, seed, base):
    keep = []
    P = port.params(cfg, keep)
    S = port.scene(nodes, bricks)
    return port.render_tile(S, P, *TILE, spp, seed=seed, sample_base=base)


def _same(g, p):
    return np.allclose(g, p, rtol=2e-5, atol=1e-6 * np.abs(p).max() + 1e-30)


def _async_tile(r, spp, seed, base):
    import torch

    from droplet_b200.renderer import stream_handle

    x0, y0, tw, th = TILE
    sun = torch.zeros((th, tw, 4), device="cuda")
    sky = torch.zeros_like(sun)
    st = torch.cuda.current_stream()
    r.render_tile_async(x0, y0, tw, th, spp, seed, base, sun.data_ptr(), sky.data_ptr(), stream_handle(st))
    st.synchronize()
    return sun.cpu().numpy(), sky.cpu().numpy()


@pytest.mark.parametrize("tuning", [(0, 8, 24, 2, 0, 3, 4), (0, 5, 16, 0, 8, 2, 1)])
def test_camera_lists_do_not_change_paths(scene, port, tuning):
    r, nodes, bricks, _ = scene
    cfg = c0_cfg(64, 64)
    r.set_params(settings_from_cfg(cfg))
    psun, psky, pcnt = _port_tile(port, cfg, nodes, bricks, 24, 13, 5)
    assert pcnt["node_visits"] > pcnt["paths"]  # the camera segments traverse nodes
    saved = r.get_tuning()
    try:
        r.set_tuning(*tuning)
        for pool in (0, N.DR_NONE, 40):  # default, no lists, most pixels' lists do not fit
            r.set_camera_lists(pool)
            for blocking in (True, False):
                r.reset_counters()
                if blocking:
                    sun, sky = r.render_tile(*TILE, 24, seed=13, sample_base=5)
                else:
                    sun, sky = _async_tile(r, 24, 13, 5)
                cnt = r.counters()
                assert _same(sun, psun) and _same(sky, psky), (tuning, pool, blocking)
                for k in KEYS:
                    assert cnt[k] == pcnt[k], (tuning, pool, blocking, k, cnt[k], pcnt[k])
    finally:
        r.set_camera_lists(0)
        r.set_tuning(*saved)


def test_sky_in_place_with_the_finiteness_check(scene, port):
    r, nodes, bricks, _ = scene
    cfg = c0_cfg(64, 64)
    cfg["finite_paths"] = True
    r.set_params(settings_from_cfg(cfg))
    psun, psky, pcnt = _port_tile(port, cfg, nodes, bricks, 24, 17, 0)
    saved = r.get_tuning()
    try:
        for tuning in [(0, 8, 24, 2, 0, 3, 4), (0, 4, 32, 0, 0, 0, 0)]:
            r.set_tuning(*tuning)
            r.reset_counters()
            sun, sky = r.render_tile(*TILE, 24, seed=17, sample_base=0)
            assert _same(sun, psun) and _same(sky, psky), tuning
            assert sky[..., :3].sum() > 0
            cnt = r.counters()
            for k in KEYS:
                assert cnt[k] == pcnt[k], (tuning, k)
    finally:
        r.set_tuning(*saved)
        r.set_params(settings_from_cfg(c0_cfg(64, 64)))


def test_batch_with_and_without_lists(scene):
    from droplet_b200.renderer import Batch, BatchView
    from droplet_b200.scene import Octree

    r, nodes, bricks, mlevel = scene
    oc = Octree(nodes, bricks, mlevel)
    views = [BatchView(0, settings_from_cfg(c0_cfg(64, 64)), 8, 100 + k) for k in range(3)]
    out = {}
    for traversal in (2, 1):  # the cell walk keeps its own traversal: no lists
        b = Batch(r, [oc], views)
        try:
            b.set_tuning(0, 8, 24, traversal, 0, 3, 2)
            b.launch()
            out[traversal] = [b.read(v) for v in range(len(views))]
        finally:
            b.close()
    for (s2, k2), (s1, k1) in zip(out[2], out[1]):
        assert _same(s2, s1) and _same(k2, k1)
        assert k2[..., :3].sum() > 0
