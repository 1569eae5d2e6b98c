"""The path-replay adjoint on the GPU: equal to the CPU restatement on the same
random streams, the transmittance gradient against the FP64 quadrature
gradient, the autograd wrapper against the direct call, and the density
gradient against central finite differences with common random numbers."""
import numpy as np
import pytest

from conftest import c0_cfg, golden_octree, settings_from_cfg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def adj():
    from droplet_b200.renderer import Renderer
    from droplet_b200.scene import Octree

    nodes, bricks, mlevel = golden_octree()
    r = Renderer(0)
    r.upload(Octree(nodes, bricks, mlevel))
    yield r, nodes, bricks
    r.close()


def _gpu_adjoint(r, cfg, x0, y0, tw, th, spp, seed, base, dsun, dsky, n_leaves):
    import torch

    r.set_params(settings_from_cfg(cfg))
    ds = torch.as_tensor(dsun, device="cuda").contiguous()
    dk = torch.as_tensor(dsky, device="cuda").contiguous()
    g = torch.zeros((n_leaves, 512), dtype=torch.float32, device="cuda")
    ga = torch.zeros(1, dtype=torch.float64, device="cuda")
    r.adjoint_tile_async(x0, y0, tw, th, spp, seed, base, ds.data_ptr(), dk.data_ptr(), g.data_ptr(), ga.data_ptr())
    torch.cuda.synchronize()
    return g.cpu().numpy().astype(np.float64), float(ga.item())


@pytest.mark.parametrize("tuning", [(0, 0, 0, 0, 0, 0, 0), (1, 0, 0, 0, 0, 0, 0)])
def test_adjoint_equals_restatement(adj, port, tuning):
    """The adjoint (whatever the forward's launch shape) equals the CPU
    restatement on the same random streams."""
    r, nodes, bricks = adj
    cfg = c0_cfg(64, 64)
    keep = []
    P = port.params(cfg, keep)
    S = port.scene(nodes, bricks)
    rng = np.random.default_rng(8)
    dsun = rng.normal(size=(40, 48, 4)).astype(np.float32)
    dsky = rng.normal(size=(40, 48, 4)).astype(np.float32)
    g_cpu, a_cpu = port.adjoint_tile(S, P, 8, 12, 48, 40, 16, 21, 3, dsun, dsky)
    saved = r.get_tuning()
    try:
        r.set_tuning(*tuning)
        g_gpu, a_gpu = _gpu_adjoint(r, cfg, 8, 12, 48, 40, 16, 21, 3, dsun, dsky, len(bricks))
    finally:
        r.set_tuning(*saved)
    scale = np.abs(g_cpu).max()
    assert scale > 0
    assert np.allclose(g_gpu, g_cpu, rtol=1e-3, atol=1e-4 * scale)
    assert (g_gpu != 0).sum() == (g_cpu != 0).sum()
    assert abs(a_gpu - a_cpu) <= 1e-4 * abs(a_cpu) + 1e-6


def test_transmittance_adjoint_equals_restatement_and_fp64(adj, port):
    import test_adjoint_oracle as T

    r, nodes, bricks = adj
    cfg = c0_cfg(8, 8)
    r.set_params(settings_from_cfg(cfg))
    keep = []
    P = port.params(cfg, keep)
    S = port.scene(nodes, bricks)
    st = cfg["sigma_s"] + cfg["sigma_a"]
    ro, rd = T._rays(nodes, 6, 4)
    w = np.linspace(0.5, 1.5, 6).astype(np.float32)
    g_gpu, T_gpu = r.adjoint_transmittance(ro.astype(np.float32), rd.astype(np.float32), w, 1 << 20, 9, len(bricks))
    g_cpu, T_cpu = port.adjoint_transmittance(S, P, ro.astype(np.float32), rd.astype(np.float32), w, 4096, 9)
    # the first 4096 samples of each ray are the CPU's: check through a small GPU run
    g_gpu_s, T_gpu_s = r.adjoint_transmittance(ro.astype(np.float32), rd.astype(np.float32), w, 4096, 9, len(bricks))
    assert np.array_equal(T_gpu_s, T_cpu)
    assert np.allclose(g_gpu_s, g_cpu, rtol=1e-4, atol=1e-6 * np.abs(g_cpu).max())
    g_ref = np.zeros_like(g_cpu)
    for i in range(6):
        tau = port.optical_depth(S, ro[i], rd[i])
        g_ref += -st * w[i] * np.exp(-st * tau) * port.optical_depth_grad(S, ro[i], rd[i])
        assert abs(T_gpu[i] - np.exp(-st * tau)) < 5e-3
    a, b = g_gpu.ravel().astype(np.float64), g_ref.ravel()
    assert abs(a @ b / (b @ b) - 1.0) < 0.01
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 0.03


def test_autograd_matches_direct_adjoint(adj):
    import torch

    from droplet_b200 import adjoint as AD

    r, nodes, bricks = adj
    cfg = c0_cfg(32, 32)
    s = settings_from_cfg(cfg)
    views = [AD.DiffView(s, 8, seed=1), AD.DiffView(s, 8, seed=2)]
    b = torch.tensor(np.asarray(bricks), device="cuda", requires_grad=True)
    albedo = torch.tensor(0.99, device="cuda", requires_grad=True)
    target = torch.rand((2, 32, 32, 4), device="cuda", generator=torch.Generator("cuda").manual_seed(0))
    sun, sky = AD.render(b, albedo, r, views, adjoint_seed_offset=0)
    loss = ((sun + sky - target)[..., :3] ** 2).sum()
    loss.backward()
    # the same adjoint through the C ABI
    d = (2 * (sun + sky - target)).detach()
    d[..., 3] = 0
    g = torch.zeros_like(b)
    ga = torch.zeros(1, dtype=torch.float64, device="cuda")
    for i, v in enumerate(views):
        r.set_params(s)
        di = (d[i] / v.spp).contiguous()
        r.adjoint_tile_async(0, 0, 32, 32, v.spp, v.seed, 0, di.data_ptr(), di.data_ptr(), g.data_ptr(), ga.data_ptr())
    torch.cuda.synchronize()
    assert torch.allclose(b.grad, g, rtol=1e-3, atol=1e-5 * float(g.abs().max()))
    assert abs(float(albedo.grad) - float(ga)) <= 1e-3 * abs(float(ga)) + 1e-6
    assert float(g.abs().max()) > 0 and float(ga) != 0


def test_density_gradient_matches_crn_finite_differences(adj):
    """Directional check on 256 random voxels: for random signs u on those
    voxels, (L(v + eps u) - L(v - eps u)) / (2 eps) with common random numbers
    and the majorants held fixed equals the adjoint's g . u; L = sum(delta *
    image) with fixed delta.  Eight independent seed groups give the spread.
    eps = 1e-2 here (the difference quotient of a delta-tracking estimator
    counts flipped decisions, so its noise falls as 1/sqrt(eps)); the C3
    check in the benchmark uses eps = 1e-3 per voxel."""
    import torch

    r, nodes, bricks = adj
    cfg = c0_cfg(48, 48)
    r.set_params(settings_from_cfg(cfg))
    nl = len(bricks)
    base = torch.tensor(np.asarray(bricks), device="cuda")
    r.set_bricks_dev(base.data_ptr(), nl, 1.05)  # headroom: majorants then stay fixed
    maj = r.majorants(len(nodes))
    leaf_of_brick = np.zeros(nl, np.int64)
    isleaf = nodes["volx"][:, 1] != 0xFFFFFFFF
    leaf_of_brick[nodes["volx"][isleaf, 1]] = np.nonzero(isleaf)[0]
    vals = np.asarray(bricks)
    eps = 1e-2
    ok = (vals + eps <= maj[leaf_of_brick][:, None]) & (vals - eps >= 0) & (vals > 0)
    cand = np.argwhere(ok.ravel()).ravel()
    rng = np.random.default_rng(5)
    pick = rng.choice(cand, 256, replace=False)
    rng2 = np.random.default_rng(6)
    dsun = torch.tensor(rng2.normal(size=(48, 48, 4)).astype(np.float32), device="cuda")
    dsky = torch.tensor(rng2.normal(size=(48, 48, 4)).astype(np.float32), device="cuda")
    spp = 32768
    sun = torch.empty((48, 48, 4), device="cuda")
    sky = torch.empty_like(sun)

    def L(b, seed):
        r.set_bricks_dev(b.data_ptr(), nl, 0.0)
        r.render_tile_async(0, 0, 48, 48, spp, seed, 0, sun.data_ptr(), sky.data_ptr())
        r.synchronize()
        return float((dsun[..., :3].double() * sun[..., :3]).sum() + (dsky[..., :3].double() * sky[..., :3]).sum())

    fds, adjs = [], []
    for k in range(8):
        u = torch.zeros(nl * 512, device="cuda")
        u[torch.as_tensor(pick, device="cuda")] = torch.as_tensor(rng.choice([-1.0, 1.0], 256).astype(np.float32),
                                                                   device="cuda")
        u = u.reshape(nl, 512)
        seed = 1000 + k
        fds.append((L(base + eps * u, seed) - L(base - eps * u, seed)) / (2 * eps))
        r.set_bricks_dev(base.data_ptr(), nl, 0.0)
        g = torch.zeros((nl, 512), device="cuda")
        ga = torch.zeros(1, dtype=torch.float64, device="cuda")
        r.adjoint_tile_async(0, 0, 48, 48, spp, seed, 0, dsun.data_ptr(), dsky.data_ptr(), g.data_ptr(), ga.data_ptr())
        torch.cuda.synchronize()
        adjs.append(float((g * u).sum()))
    fds, adjs = np.array(fds), np.array(adjs)
    diff = fds - adjs
    print("fd", fds, "adjoint", adjs)
    assert abs(diff.mean()) < 4 * diff.std(ddof=1) / np.sqrt(8) + 1e-9, (fds, adjs)
    # the check has power: the directional derivatives stand well above the FD-adjoint spread
    assert np.sqrt((adjs ** 2).mean()) > 2 * diff.std(ddof=1), (fds, adjs)


def test_sky_zero_over_zero_path_on_gpu(port):
    """The reference's NaN sky path (rd.y == 0 at escape) is reproduced bit for
    bit on the GPU; DR_KERNEL_FINITE_PATHS drops it in every kernel family."""
    from conftest import NAN_PATH, orbit_cfg, uniform_cube_scene
    from droplet_b200.renderer import Renderer
    from droplet_b200.scene import Octree, build_octree

    oc = uniform_cube_scene(lambda o, v, s, d: build_octree(o, v, s, d))
    cfg = orbit_cfg(256, 256, 0.0)
    px, py = NAN_PATH["pixel"]
    with Renderer(0) as r:
        r.upload(oc)
        r.set_params(settings_from_cfg(cfg))
        sun, sky = r.probe_paths([px], [py], [NAN_PATH["sample"]], NAN_PATH["seed"])
        assert np.isnan(sky[0, :3]).all()
        cfg["finite_paths"] = True
        r.set_params(settings_from_cfg(cfg))
        sun, sky = r.probe_paths([px], [py], [NAN_PATH["sample"]], NAN_PATH["seed"])
        assert (sky[0, :3] == 0).all() and (sun[0, :3] == 0).all()
        for tuning in ((1, 0, 0, 0, 0), (0, 5, 24, 0, 0), (0, 8, 24, 1, 8)):
            r.set_tuning(*tuning)
            a, b = r.render_tile(px - 1, py, 2, 2, 16, seed=NAN_PATH["seed"], sample_base=0)
            assert np.isfinite(a).all() and np.isfinite(b).all(), tuning


def test_autograd_on_default_stream_matches_render(adj):
    """The autograd wrapper launches on torch's current stream (the default one
    here): its images equal a blocking render of the same paths, and its albedo
    gradient is not empty."""
    import torch

    from droplet_b200 import adjoint as AD

    r, nodes, bricks = adj
    cfg = c0_cfg(256, 256)
    cfg["finite_paths"] = True
    s = settings_from_cfg(cfg)
    b = torch.tensor(np.asarray(bricks), device="cuda", requires_grad=True)
    albedo = torch.tensor(0.99, device="cuda", requires_grad=True)
    sun, sky = AD.render(b, albedo, r, [AD.DiffView(s, 64, seed=11)])
    got = (sun[0] + sky[0]).detach().cpu().numpy()
    r.set_params(AD._with_albedo(s, 0.99))
    ps, pk = r.render_tile(0, 0, 256, 256, 64, seed=11, sample_base=0)
    ref = (ps + pk) / 64
    assert np.allclose(got, ref, rtol=1e-5, atol=1e-6 * np.abs(ref).max())
    (sun + sky)[..., :3].sum().backward()
    assert float(albedo.grad) != 0.0 and float(b.grad.abs().sum()) > 0


def test_reweighted_loss_equals_restatement_and_differences_match_adjoint(adj, port):
    """dr_reweighted_loss_async equals the CPU restatement on the same streams,
    and its central differences (eps 1e-3, common random numbers) along random
    signs on 256 brick samples equal the adjoint's directional derivative."""
    import torch

    r, nodes, bricks = adj
    cfg = c0_cfg(64, 64)
    keep = []
    P = port.params(cfg, keep)
    S = port.scene(nodes, bricks)
    rng = np.random.default_rng(12)
    tw, th, spp, seed = 48, 40, 16, 23
    dsun = rng.normal(size=(th, tw, 4)).astype(np.float32)
    dsky = rng.normal(size=(th, tw, 4)).astype(np.float32)
    base = np.asarray(bricks, np.float32).reshape(-1, 512)
    flat = base.reshape(-1)
    pick = rng.choice(np.flatnonzero(flat >= 0.05), 256, replace=False)
    u = np.zeros(flat.size, np.float32)
    u[pick] = rng.choice([-1.0, 1.0], 256)
    u = u.reshape(base.shape)
    eps = 1e-3
    r.set_params(settings_from_cfg(cfg))
    ds = torch.as_tensor(dsun, device="cuda").contiguous()
    dk = torch.as_tensor(dsky, device="cuda").contiguous()

    def gpu_loss(pert):
        pt = torch.as_tensor(np.ascontiguousarray(pert, np.float32), device="cuda")
        out = torch.zeros(1, dtype=torch.float64, device="cuda")
        r.reweighted_loss_async(8, 12, tw, th, spp, seed, 3, ds.data_ptr(), dk.data_ptr(), pt.data_ptr(),
                                out.data_ptr())
        torch.cuda.synchronize()
        return float(out.item())

    lp = gpu_loss(base + eps * u)
    lp_cpu = port.reweighted_loss(S, P, 8, 12, tw, th, spp, seed, 3, dsun, dsky, base + eps * u)
    assert abs(lp - lp_cpu) <= 1e-6 * abs(lp_cpu)
    lm = gpu_loss(base - eps * u)
    g, _ = _gpu_adjoint(r, cfg, 8, 12, tw, th, spp, seed, 3, dsun, dsky, len(bricks))
    fd = (lp - lm) / (2 * eps)
    ad = float((g * u).sum())
    assert abs(ad) > 0
    assert abs(fd - ad) <= 1e-3 * abs(ad), (fd, ad)


def test_adjoint_across_path_chunks_equals_two_halves(adj):
    """A 512x512 tile at 40 spp has 10.5 M paths, more than one chunk of the
    totals/scatter passes (2^23 paths): its gradient equals the sum of the two
    20-spp halves (sample_base 0 and 20), each within one chunk, up to the
    order of the float atomics."""
    import torch

    r, nodes, bricks = adj
    cfg = c0_cfg(512, 512)
    r.set_params(settings_from_cfg(cfg))
    rng = np.random.default_rng(13)
    d = torch.as_tensor(rng.normal(size=(512, 512, 4)).astype(np.float32) * 1e-3, device="cuda").contiguous()

    def grad(spp, base):
        g = torch.zeros((len(bricks), 512), dtype=torch.float32, device="cuda")
        ga = torch.zeros(1, dtype=torch.float64, device="cuda")
        r.adjoint_tile_async(0, 0, 512, 512, spp, 31, base, d.data_ptr(), d.data_ptr(), g.data_ptr(), ga.data_ptr())
        torch.cuda.synchronize()
        return g.double().cpu().numpy(), float(ga.item())

    g_full, a_full = grad(40, 0)
    g_a, a_a = grad(20, 0)
    g_b, a_b = grad(20, 20)
    scale = np.abs(g_full).max()
    assert scale > 0
    assert np.allclose(g_full, g_a + g_b, rtol=1e-4, atol=1e-5 * scale)
    assert abs(a_full - (a_a + a_b)) <= 1e-5 * abs(a_full)
