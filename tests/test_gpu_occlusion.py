"""Holdout-mesh occlusion on the GPU (the occluder BVH and its any-hit
traversal in place of Embree, src/SceneOcclusion.cpp:19-91) against the CPU
restatement, which tests every triangle: the hit answer per ray bit-exact
(random rays, rays aimed at vertices and edges, rays leaving an occluder's
surface), and the USE_EMBREE build's render semantics in every kernel: path
samples bit-exact, tiles of every launch shape, the shadow pass, depth
compositing and the adjoint."""
import numpy as np
import pytest

from conftest import c0_cfg, depth_texture, golden_octree, occluder_surfaces, settings_from_cfg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def occ_renderer():
    from droplet_b200.renderer import Renderer
    from droplet_b200.scene import Octree

    nodes, bricks, mlevel = golden_octree()
    r = Renderer(0)
    r.set_occluders(occluder_surfaces())  # before the scene: kept across the upload
    r.upload(Octree(nodes, bricks, mlevel))
    yield r
    r.close()


class _OccScene:
    """The restatement's scene with occluders; holds the arrays its raw pointers refer to."""

    def __init__(self, port):
        self.nodes, self.bricks, _ = golden_octree()
        self.occ = port.occluder_triangles(occluder_surfaces(), 0)
        self.S = port.scene(self.nodes, self.bricks, self.occ)

    def __iter__(self):
        return iter((self.S, self.occ))


@pytest.fixture(scope="module")
def occ_scene(port):
    return _OccScene(port)


def _probe_rays(occ, n, seed):
    rng = np.random.default_rng(seed)
    ro = rng.uniform([-0.5, -0.5, 0.1], [2.0, 2.0, 1.5], (n, 3))
    rd = rng.normal(size=(n, 3))
    # aimed at vertices and edge points of random triangles
    k = rng.integers(0, len(occ), n)
    t = occ[k].astype(np.float64)
    # (a, b) of v0 + a e1 + b e2: the three vertices and the three edge midpoints
    ab = np.array([[0, 0], [1, 0], [0, 1], [0.5, 0], [0, 0.5], [0.5, 0.5]])[rng.integers(0, 6, n)]
    tgt = t[:, 0:3] + ab[:, :1] * t[:, 4:7] + ab[:, 1:] * t[:, 8:11]
    aim = rng.random(n) < 0.4
    rd[aim] = tgt[aim] - ro[aim]
    # leaving an occluder's surface (origin on a triangle, t = 0 hits count)
    on = rng.random(n) < 0.15
    b = rng.dirichlet([1, 1, 1], n)
    ro[on] = (t[:, 0:3] + b[:, 1:2] * t[:, 4:7] + b[:, 2:3] * t[:, 8:11])[on]
    rd /= np.linalg.norm(rd, axis=1, keepdims=True)
    return ro.astype(np.float32), rd.astype(np.float32)


def test_occlusion_probe_equals_restatement(occ_renderer, occ_scene, port):
    S, occ = occ_scene
    ro, rd = _probe_rays(occ, 6000, 5)
    gpu = occ_renderer.probe_occlusion(ro, rd)
    cpu = port.occluded(S, ro, rd)
    assert np.array_equal(gpu, cpu)
    assert 0.05 < gpu.mean() < 0.95


def test_holdout_only_occluders_equal_restatement(port):
    from droplet_b200.renderer import OCCLUDE_HOLDOUT_ONLY, Renderer

    nodes, bricks, _ = golden_octree()
    surfaces = occluder_surfaces()
    occ = port.occluder_triangles(surfaces, 1)
    S = port.scene(nodes, bricks, occ)
    with Renderer(0) as r:
        r.set_occluders(surfaces, OCCLUDE_HOLDOUT_ONLY)
        ro, rd = _probe_rays(occ, 3000, 6)
        assert np.array_equal(r.probe_occlusion(ro, rd), port.occluded(S, ro, rd))
        r.set_occluders([])
        assert not r.probe_occlusion(ro, rd).any()


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_path_samples_with_occluders_bit_exact(occ_renderer, occ_scene, port):
    S, _ = occ_scene
    cfg = c0_cfg(64, 64)
    cfg["embree"] = True
    keep = []
    P = port.params(cfg, keep)
    occ_renderer.set_params(settings_from_cfg(cfg))
    rng = np.random.default_rng(13)
    n = 3000
    px = rng.integers(16, 48, n).astype(np.uint32)
    py = rng.integers(20, 44, n).astype(np.uint32)
    sm = rng.integers(0, 1 << 40, n).astype(np.uint64)
    a, b = occ_renderer.probe_paths(px, py, sm, seed=78)
    for i in range(n):
        pa, pb, _ = port.render_path(S, P, int(px[i]), int(py[i]), 78, int(sm[i]))
        assert np.array_equal(bits(a[i]), bits(pa)), (i, a[i], pa)
        assert np.array_equal(bits(b[i]), bits(pb)), (i, b[i], pb)


@pytest.mark.parametrize("tuning", [(0, 0, 0, 0, 0, 0, 0), (1, 0, 0, 0, 0, 0, 0), (0, 8, 24, 0, 8, 4, 4),
                                    (0, 5, 8, 1, 0, 0, 0)])
def test_tiles_with_occluders_equal_restatement(occ_renderer, occ_scene, port, tuning):
    S, _ = occ_scene
    nodes, bricks, _ = golden_octree()
    cfg = c0_cfg(64, 64)
    cfg["embree"] = True
    keep = []
    P = port.params(cfg, keep)
    occ_renderer.set_params(settings_from_cfg(cfg))
    saved = occ_renderer.get_tuning()
    try:
        occ_renderer.set_tuning(*tuning)
        sun, sky = occ_renderer.render_tile(8, 10, 48, 44, 32, seed=5, sample_base=0)
    finally:
        occ_renderer.set_tuning(*saved)
    psun, psky, _ = port.render_tile(S, P, 8, 10, 48, 44, 32, seed=5, sample_base=0)
    for g, p in ((sun, psun), (sky, psky)):
        assert np.allclose(g, p, rtol=2e-5, atol=1e-6 * np.abs(p).max() + 1e-30), tuning
    # the occluders take light away
    bsun, bsky, _ = port.render_tile(port.scene(nodes, bricks), P, 8, 10, 48, 44, 32, seed=5, sample_base=0)
    assert sun[..., :3].sum() < 0.97 * bsun[..., :3].sum() and sky[..., :3].sum() < 0.97 * bsky[..., :3].sum()


def test_depth_cut_alpha_in_embree_build_equals_restatement(occ_renderer, occ_scene, port):
    S, _ = occ_scene
    cfg = c0_cfg(64, 64)
    cfg["depth"] = depth_texture(64, 64)
    cfg["depthcomp"] = True
    cfg["embree"] = True
    keep = []
    P = port.params(cfg, keep)
    occ_renderer.set_params(settings_from_cfg(cfg))
    sun, sky = occ_renderer.render_tile(4, 6, 56, 52, 24, seed=8, sample_base=0)
    psun, psky, _ = port.render_tile(S, P, 4, 6, 56, 52, 24, seed=8, sample_base=0)
    for g, p in ((sun, psun), (sky, psky)):
        assert np.allclose(g, p, rtol=2e-5, atol=1e-6 * np.abs(p).max() + 1e-30)


def test_shadow_pass_with_occluders_equals_restatement(occ_renderer, occ_scene, port):
    """rgb bit for bit; alpha +inf, or NaN (0/0) where a sample's sun ray was
    occluded."""
    S, _ = occ_scene
    cfg = c0_cfg(64, 64)
    cfg["depth"] = depth_texture(64, 64)
    cfg["embree"] = True
    keep = []
    P = port.params(cfg, keep)
    occ_renderer.set_params(settings_from_cfg(cfg))
    x0, y0, tw, th, spp = 6, 4, 50, 54, 64
    ref, _ = port.shadow_tile(S, P, x0, y0, tw, th, spp, seed=22, sample_base=1)
    got, _ = occ_renderer.render_shadow_tile(x0, y0, tw, th, spp, seed=22, sample_base=1)
    assert np.array_equal(got[..., :3], ref[..., :3])
    assert np.array_equal(np.isnan(got[..., 3]), np.isnan(ref[..., 3]))
    assert np.isnan(got[..., 3]).any()  # some sun rays hit the sphere
    assert np.isposinf(got[..., 3][~np.isnan(got[..., 3])]).all()


def test_adjoint_with_occluders_equals_restatement(occ_renderer, occ_scene, port):
    import torch

    S, _ = occ_scene
    nodes, bricks, _ = golden_octree()
    cfg = c0_cfg(64, 64)
    cfg["embree"] = True
    keep = []
    P = port.params(cfg, keep)
    rng = np.random.default_rng(9)
    dsun = rng.normal(size=(40, 48, 4)).astype(np.float32)
    dsky = rng.normal(size=(40, 48, 4)).astype(np.float32)
    g_cpu, a_cpu = port.adjoint_tile(S, P, 8, 12, 48, 40, 16, 21, 3, dsun, dsky)
    occ_renderer.set_params(settings_from_cfg(cfg))
    ds = torch.as_tensor(dsun, device="cuda").contiguous()
    dk = torch.as_tensor(dsky, device="cuda").contiguous()
    g = torch.zeros((len(bricks), 512), dtype=torch.float32, device="cuda")
    ga = torch.zeros(1, dtype=torch.float64, device="cuda")
    occ_renderer.adjoint_tile_async(8, 12, 48, 40, 16, 21, 3, ds.data_ptr(), dk.data_ptr(), g.data_ptr(),
                                    ga.data_ptr())
    torch.cuda.synchronize()
    g_gpu = g.cpu().numpy().astype(np.float64)
    scale = np.abs(g_cpu).max()
    assert scale > 0
    assert np.allclose(g_gpu, g_cpu, rtol=1e-3, atol=1e-4 * scale)
    assert abs(float(ga.item()) - a_cpu) <= 1e-4 * abs(a_cpu) + 1e-6
