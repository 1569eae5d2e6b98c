"""Surface (SDF) leaves on the GPU against the CPU restatement (pinned to the
compiled reference in test_sdf): path samples bit-exact, tiles of every launch
shape, the shadow pass, a batch and the adjoint."""
import numpy as np
import pytest

from conftest import c0_cfg, depth_texture, sdf_scene, settings_from_cfg

pytestmark = pytest.mark.gpu


class _Scene:
    def __init__(self, port):
        self.nodes, self.bricks, self.sdf, self.mlevel = sdf_scene()
        self.S = port.scene(self.nodes, self.bricks, None, self.sdf)

    def octree(self):
        from droplet_b200.scene import Octree

        return Octree(self.nodes, self.bricks, self.mlevel, self.sdf)


@pytest.fixture(scope="module")
def scene(port):
    return _Scene(port)


@pytest.fixture(scope="module")
def renderer(scene):
    from droplet_b200.renderer import Renderer

    r = Renderer(0)
    r.upload(scene.octree())
    yield r
    r.close()


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_path_samples_bit_exact(renderer, scene, port):
    cfg = c0_cfg(64, 64)
    renderer.set_params(settings_from_cfg(cfg))
    keep = []
    P = port.params(cfg, keep)
    rng = np.random.default_rng(15)
    n = 3000
    px = rng.integers(16, 48, n).astype(np.uint32)
    py = rng.integers(20, 44, n).astype(np.uint32)
    sm = rng.integers(0, 1 << 40, n).astype(np.uint64)
    a, b = renderer.probe_paths(px, py, sm, seed=80)
    opaque = 0
    for i in range(n):
        pa, pb, _ = port.render_path(scene.S, P, int(px[i]), int(py[i]), 80, int(sm[i]))
        assert np.array_equal(bits(a[i]), bits(pa)), (i, a[i], pa)
        assert np.array_equal(bits(b[i]), bits(pb)), (i, b[i], pb)
        opaque += pa[3] > 0
    assert opaque > 300


@pytest.mark.parametrize("tuning", [(0, 0, 0, 0, 0, 0, 0), (1, 0, 0, 0, 0, 0, 0), (0, 8, 24, 0, 8, 4, 4),
                                    (0, 5, 8, 1, 0, 0, 0)])
def test_tiles_equal_restatement(renderer, scene, port, tuning):
    cfg = c0_cfg(64, 64)
    renderer.set_params(settings_from_cfg(cfg))
    keep = []
    P = port.params(cfg, keep)
    saved = renderer.get_tuning()
    try:
        renderer.set_tuning(*tuning)
        renderer.reset_counters()
        sun, sky = renderer.render_tile(8, 10, 48, 44, 32, seed=6, sample_base=0)
        cnt = renderer.counters()
    finally:
        renderer.set_tuning(*saved)
    psun, psky, pcnt = port.render_tile(scene.S, P, 8, 10, 48, 44, 32, seed=6, sample_base=0)
    for g, p in ((sun, psun), (sky, psky)):
        assert np.allclose(g, p, rtol=2e-5, atol=1e-6 * np.abs(p).max() + 1e-30), tuning
    for k in ("vertices", "density_lookups", "paths"):
        assert cnt[k] == pcnt[k], (tuning, k, cnt[k], pcnt[k])


def test_shadow_pass_equals_restatement(renderer, scene, port):
    cfg = c0_cfg(64, 64)
    cfg["depth"] = depth_texture(64, 64)
    renderer.set_params(settings_from_cfg(cfg))
    keep = []
    P = port.params(cfg, keep)
    ref, _ = port.shadow_tile(scene.S, P, 6, 4, 50, 54, 48, seed=23, sample_base=2)
    got, _ = renderer.render_shadow_tile(6, 4, 50, 54, 48, seed=23, sample_base=2)
    assert np.array_equal(got[..., :3], ref[..., :3])


def test_batch_with_surface_scene_equals_restatement(scene, port):
    from droplet_b200.renderer import Batch, BatchView, Renderer
    from droplet_b200.scene import Octree
    from conftest import golden_octree

    nodes0, bricks0, mlevel0 = golden_octree()
    cfg = c0_cfg(64, 64)
    with Renderer(0) as r:
        b = Batch(r, [Octree(nodes0, bricks0, mlevel0), scene.octree()],
                  [BatchView(0, settings_from_cfg(cfg), 16, 7), BatchView(1, settings_from_cfg(cfg), 16, 8)])
        try:
            b.launch()
            outs = [b.read(v) for v in range(2)]
        finally:
            b.close()
    keep = []
    P = port.params(cfg, keep)
    S0 = port.scene(nodes0, bricks0)
    for v, (S, seed) in enumerate(((S0, 7), (scene.S, 8))):
        psun, psky, _ = port.render_tile(S, P, 0, 0, 64, 64, 16, seed=seed, sample_base=0)
        for g, p in zip(outs[v], (psun, psky)):
            assert np.allclose(g, p, rtol=2e-5, atol=1e-6 * np.abs(p).max() + 1e-30), v


def test_adjoint_equals_restatement(renderer, scene, port):
    import torch

    cfg = c0_cfg(64, 64)
    keep = []
    P = port.params(cfg, keep)
    rng = np.random.default_rng(11)
    dsun = rng.normal(size=(40, 48, 4)).astype(np.float32)
    dsky = rng.normal(size=(40, 48, 4)).astype(np.float32)
    g_cpu, a_cpu = port.adjoint_tile(scene.S, P, 8, 12, 48, 40, 16, 21, 3, dsun, dsky)
    renderer.set_params(settings_from_cfg(cfg))
    ds = torch.as_tensor(dsun, device="cuda").contiguous()
    dk = torch.as_tensor(dsky, device="cuda").contiguous()
    g = torch.zeros((len(scene.bricks), 512), dtype=torch.float32, device="cuda")
    ga = torch.zeros(1, dtype=torch.float64, device="cuda")
    renderer.adjoint_tile_async(8, 12, 48, 40, 16, 21, 3, ds.data_ptr(), dk.data_ptr(), g.data_ptr(), ga.data_ptr())
    torch.cuda.synchronize()
    g_gpu = g.cpu().numpy().astype(np.float64)
    scale = np.abs(g_cpu).max()
    assert scale > 0
    assert np.allclose(g_gpu, g_cpu, rtol=1e-3, atol=1e-4 * scale)
    assert abs(float(ga.item()) - a_cpu) <= 1e-4 * abs(a_cpu) + 1e-6
