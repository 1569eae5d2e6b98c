"""GPU parity: the CUDA path (through the C ABI) against the reference's
golden vectors, the compiled reference where present, and the CPU
restatement.

Bars (written into each test):
  * octree leaf sequences and (tr0, tr1), brick lookups, Mie table lookups: bit-exact;
  * whole path samples against the CPU restatement on the same streams: bit-exact;
  * images against the reference: relative bias <= 1% after removing the
    reference's own Monte Carlo noise (two independent 65536-spp runs);
  * transmittance against FP64 quadrature: <= 1e-4 relative.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import c0_cfg, golden, golden_octree, settings_from_cfg
from droplet_b200 import _native as N

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def same_floats(a, b):
    """Bit-identical, except that any NaN matches any NaN: exactly axis-parallel
    rays give NaN intervals on both sides, and the host's default NaN (sign bit
    set) differs from the device's canonical NaN."""
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    nan = np.isnan(a) & np.isnan(b)
    return a.shape == b.shape and bool(((a.view(np.uint32) == b.view(np.uint32)) | nan).all())


def test_leaf_sequences_bit_exact_vs_reference_vectors(gpu_renderer):
    z = golden("ref_leaf_sequences.npz")
    maxn = z["nodes"].shape[1]
    nodes, a, b, cnt = gpu_renderer.probe_leaf_sequence(z["ro"], z["rd"], maxn)
    assert np.array_equal(cnt, z["count"])
    for i in range(len(cnt)):
        k = int(cnt[i])
        assert np.array_equal(nodes[i, :k], z["nodes"][i, :k])
        assert same_floats(a[i, :k], z["tr0"][i, :k])
        assert same_floats(b[i, :k], z["tr1"][i, :k])


def test_leaf_sequences_bit_exact_vs_port_random_rays(gpu_renderer, port):
    onodes, _, _ = golden_octree()
    rng = np.random.default_rng(99)
    n = 20000
    ro = np.where(rng.random((n, 1)) < 0.5, rng.uniform(-1.5, 2.5, (n, 3)), rng.uniform(0.1, 0.9, (n, 3)))
    rd = rng.normal(size=(n, 3))
    rd[:30] = np.eye(3)[np.arange(30) % 3] * np.where(np.arange(30) % 2, 1, -1)[:, None]
    ro = ro.astype(np.float32)
    rd = (rd / np.linalg.norm(rd, axis=1, keepdims=True)).astype(np.float32)
    nodes, a, b, cnt = gpu_renderer.probe_leaf_sequence(ro, rd, 64)
    for i in range(n):
        pn, pa, pb = port.leaf_sequence(onodes, ro[i], rd[i], 64)
        k = int(cnt[i])
        assert k == len(pn)
        assert np.array_equal(nodes[i, :k], pn)
        assert same_floats(a[i, :k], pa) and same_floats(b[i, :k], pb)


def _degenerate_rays(nodes, rng, n_random=4000):
    """Rays that hit exact plane intersections: origins on leaf-cell corners,
    edges and the root centre, diagonal and nearly axis-aligned directions."""
    c = nodes["ce"][0][:3].astype(np.float64)
    e = float(nodes["ce"][0][3])
    leaf = nodes[nodes["volx"][:, 1] != 0xFFFFFFFF]
    cell = 2.0 * float(leaf["ce"][0][3])
    ro, rd = [], []
    dirs = [(1, 1, 1), (1, 1, 0.5), (1, 0.5, 0.25), (-1, 1, 1), (1, -1, 1), (1, 1, -1), (-1, -1, -1), (1, 2, 4),
            (2, 1, 1e-7), (1e-6, 1, 1), (1, 1e-6, 1e-6), (3, 2, 1)]
    corners = [c, c - e, c - e + cell, c + 0.5 * cell, c - 0.25 * e]
    for o in corners:
        for d in dirs:
            for back in (0.0, 1.5):
                dd = np.asarray(d, np.float64)
                dd = dd / np.linalg.norm(dd)
                ro.append(o - back * dd)
                rd.append(dd)
    # random origins snapped to the leaf-cell lattice, random directions
    k = rng.integers(-2, int(2 * e / cell) + 3, (n_random, 3))
    o = (c - e) + k * cell
    d = rng.normal(size=(n_random, 3))
    ro += list(o)
    rd += list(d / np.linalg.norm(d, axis=1, keepdims=True))
    return np.asarray(ro, np.float32), np.asarray(rd, np.float32)


@pytest.mark.parametrize("scene", ["c0", "cumulus128"])
def test_cell_walk_matches_stack_traversal_on_degenerate_rays(port, scene):
    """The GPU cell walk reports the same leaves and (tr0, tr1) as the
    reference's stack traversal (CPU restatement), on rays through exact
    plane intersections, for a depth-2 and a depth-4 leaf grid."""
    from droplet_b200 import workloads as W
    from droplet_b200.renderer import Renderer
    from droplet_b200.scene import Octree, build_octree

    if scene == "c0":
        nodes, bricks, mlevel = golden_octree()
        oc = Octree(nodes, bricks, mlevel)
    else:
        rec = W.cumulus_recipe(128)
        org, vals = W.sparse_field(rec)
        oc = build_octree(org, vals, rec.voxel_size, 12)
    rng = np.random.default_rng(5)
    ro, rd = _degenerate_rays(oc.nodes, rng)
    with Renderer(0) as r:
        r.upload(oc)
        r.set_params(settings_from_cfg(c0_cfg(64, 64)))
        nodes_g, a, b, cnt = r.probe_leaf_sequence(ro, rd, 512)
    for i in range(len(ro)):
        pn, pa, pb = port.leaf_sequence(oc.nodes, ro[i], rd[i], 512)
        k = int(cnt[i])
        assert k == len(pn), (i, ro[i], rd[i], k, len(pn))
        assert np.array_equal(nodes_g[i, :k], pn), (i, ro[i], rd[i])
        assert same_floats(a[i, :k], pa) and same_floats(b[i, :k], pb), (i, ro[i], rd[i])


def test_brick_lookup_bit_exact_vs_reference_vectors(gpu_renderer):
    z = golden("ref_samplers.npz")
    got = gpu_renderer.probe_density(z["leaf"], z["pts"])
    assert np.array_equal(bits(got), bits(z["density"]))


def test_mie_evaluate_bit_exact_vs_reference_vectors(gpu_renderer):
    z = golden("ref_samplers.npz")
    got = gpu_renderer.probe_sampler(N.DR_PROBE_MIE_EVAL_RGB, z["ct"], len(z["ct"]))
    assert np.array_equal(bits(got), bits(z["mie_rgb"]))


def test_mie_and_sun_sampling_vs_reference_vectors_and_port(gpu_renderer, port):
    z = golden("ref_samplers.npz")
    n = len(z["u1"])
    inp = np.concatenate([z["iv"].ravel(), z["u1"], z["u2"]])
    mie = gpu_renderer.probe_sampler(N.DR_PROBE_MIE_SAMPLE, inp, n)
    assert np.abs(mie - z["mie_dir"]).max() < 4e-6  # sin/cos: ulp-level vs the reference's SSE versions
    sun = gpu_renderer.probe_sampler(N.DR_PROBE_SUN_SAMPLE, np.concatenate([z["u1"], z["u2"]]), n)
    assert np.abs(sun - z["sun_dir"]).max() < 2e-6
    keep = []
    P = port.params(c0_cfg(64, 64), keep)
    d = np.zeros(3, np.float32)
    for i in range(n):
        port.L.orc_mie_sample(C.byref(P), z["iv"][i].ctypes.data, float(z["u1"][i]), float(z["u2"][i]), d.ctypes.data)
        assert np.array_equal(bits(mie[i]), bits(d))
        port.L.orc_sun_sample(C.byref(P), float(z["u1"][i]), float(z["u2"][i]), d.ctypes.data)
        assert np.array_equal(bits(sun[i]), bits(d))


def test_mie_theta_equals_reference_scan(gpu_renderer, port):
    keep = []
    P = port.params(c0_cfg(64, 64), keep)
    rng = np.random.default_rng(4)
    u = np.concatenate([rng.random(100000), np.linspace(0, 1, 30001)[1:-1]]).astype(np.float32)
    th = gpu_renderer.probe_sampler(N.DR_PROBE_MIE_THETA, u, len(u))
    scan = np.array([port.L.orc_mie_sample_theta_scan(C.byref(P), float(x)) for x in u], np.float32)
    assert np.array_equal(bits(th), bits(scan))


def test_sky_bit_exact_vs_port(gpu_renderer, port):
    keep = []
    P = port.params(c0_cfg(64, 64), keep)
    rng = np.random.default_rng(8)
    n = 20000
    rd = rng.normal(size=(n, 3))
    rd = (rd / np.linalg.norm(rd, axis=1, keepdims=True)).astype(np.float32)
    got = gpu_renderer.probe_sampler(N.DR_PROBE_SKY, rd, n)
    out = np.zeros(3, np.float32)
    for i in range(n):
        port.L.orc_sky_eval(C.byref(P), rd[i].ctypes.data, out.ctypes.data)
        assert np.array_equal(bits(got[i]), bits(out)), (i, got[i], out)


def test_path_samples_bit_exact_vs_port(gpu_renderer, port):
    """Same PCG32 stream per (seed, pixel, sample) and the same binary32 operations:
    every path sample (sun rgba, sky rgba) is bit-identical to the CPU restatement."""
    nodes, bricks, _ = golden_octree()
    cfg = c0_cfg(64, 64)
    keep = []
    P = port.params(cfg, keep)
    S = port.scene(nodes, bricks)
    rng = np.random.default_rng(12)
    n = 6000
    px = rng.integers(16, 48, n).astype(np.uint32)
    py = rng.integers(20, 44, n).astype(np.uint32)
    sm = rng.integers(0, 1 << 40, n).astype(np.uint64)
    a, b = gpu_renderer.probe_paths(px, py, sm, seed=77)
    hits = 0
    for i in range(n):
        pa, pb, cnt = port.render_path(S, P, int(px[i]), int(py[i]), 77, int(sm[i]))
        assert np.array_equal(bits(a[i]), bits(pa)), (i, a[i], pa)
        assert np.array_equal(bits(b[i]), bits(pb)), (i, b[i], pb)
        hits += pa[3] > 0
    assert hits > 200  # the sample set exercises scattering paths


def test_tile_render_matches_port_tile(gpu_renderer, port):
    nodes, bricks, _ = golden_octree()
    cfg = c0_cfg(64, 64)
    keep = []
    P = port.params(cfg, keep)
    S = port.scene(nodes, bricks)
    sun, sky = gpu_renderer.render_tile(8, 10, 48, 44, 64, seed=5, sample_base=0)
    psun, psky, _ = port.render_tile(S, P, 8, 10, 48, 44, 64, seed=5, sample_base=0)
    # identical paths; only the order of the per-pixel float sums differs
    for g, p in ((sun, psun), (sky, psky)):
        assert np.allclose(g, p, rtol=2e-5, atol=1e-6 * np.abs(p).max() + 1e-30)


def test_every_launch_shape_renders_the_same_paths(gpu_renderer, port):
    """Persistent kernel variants (blocks per SM, event batch, stack traversal
    with its stack in local or shared memory, or cell walk) and the
    one-thread-per-path kernel trace identical paths: tiles
    agree with the CPU restatement up to summation order, and the path counters
    agree exactly.  Node visits are compared for the stack traversals only: the
    cell walk visits grid cells, not octree nodes."""
    nodes, bricks, _ = golden_octree()
    cfg = c0_cfg(64, 64)
    keep = []
    P = port.params(cfg, keep)
    S = port.scene(nodes, bricks)
    psun, psky, pcnt = port.render_tile(S, P, 4, 6, 56, 52, 40, seed=9, sample_base=3)
    saved = gpu_renderer.get_tuning()
    try:
        for cand in [(0, 4, 1, 0), (0, 5, 8, 0), (0, 6, 16, 0), (0, 8, 32, 0), (0, 0, 0, 0),
                     (0, 4, 1, 1), (0, 5, 8, 1), (0, 6, 16, 1), (0, 8, 32, 1), (1, 0, 0, 0),
                     (0, 5, 8, 0, 0, 1), (0, 8, 24, 0, 8, 2, 2), (0, 6, 16, 0, 16, 4, 4),
                     (0, 4, 8, 2), (0, 5, 24, 2, 0, 3, 2), (0, 6, 16, 2, 8, 0, 4), (0, 8, 24, 2, 16, 4, 1)]:
            gpu_renderer.set_tuning(*cand)
            gpu_renderer.reset_counters()
            sun, sky = gpu_renderer.render_tile(4, 6, 56, 52, 40, seed=9, sample_base=3)
            cnt = gpu_renderer.counters()
            for g, p in ((sun, psun), (sky, psky)):
                assert np.allclose(g, p, rtol=2e-5, atol=1e-6 * np.abs(p).max() + 1e-30), cand
            keys = ("vertices", "density_lookups", "mie_evals", "paths") + (("node_visits",) if cand[3] != 1 else ())
            for k in keys:
                assert cnt[k] == pcnt[k], (cand, k, cnt[k], pcnt[k])
    finally:
        gpu_renderer.set_tuning(*saved)


def test_tuning_values_are_checked(gpu_renderer):
    """dr_set_tuning takes traversal 0 (stack, local memory), 1 (cell walk) and
    2 (stack, shared memory) and refuses anything else without changing the
    context's launch shape."""
    from droplet_b200._native import DrError

    saved = gpu_renderer.get_tuning()
    try:
        gpu_renderer.set_tuning(0, 8, 24, 2, 0, 3, 2)
        assert gpu_renderer.get_tuning() == (0, 8, 24, 2, 0, 3, 2)
        with pytest.raises(DrError):
            gpu_renderer.set_tuning(0, 8, 24, 3, 0, 3, 2)
        assert gpu_renderer.get_tuning() == (0, 8, 24, 2, 0, 3, 2)
    finally:
        gpu_renderer.set_tuning(*saved)


def _rel(x, y):
    return float(np.sqrt(((x - y) ** 2).sum()) / np.sqrt((y ** 2).sum()))


def test_image_parity_vs_reference_renders():
    """Config 0 at 128x128: GPU at 2^18 spp against two independent, converged
    reference renders at 65536 spp.  The reference's own noise is measured from A vs B;
    the remaining relative bias must stay within 1% for both buffers."""
    from droplet_b200.renderer import Renderer
    from droplet_b200.scene import Octree

    z = golden("ref_c0_images.npz")
    spp_ref = int(z["spp"].reshape(-1)[0])
    w = int(z["w"].reshape(-1)[0])
    nodes, bricks, mlevel = golden_octree()
    with Renderer(0) as r:
        r.upload(Octree(nodes, bricks, mlevel))
        r.set_params(settings_from_cfg(c0_cfg(w, w)))
        spp_g = 1 << 18
        sun = np.zeros((w, w, 4), np.float64)
        sky = np.zeros((w, w, 4), np.float64)
        for k in range(spp_g // 16384):
            a, b = r.render_tile(0, 0, w, w, 16384, seed=2024, sample_base=k * 16384)
            sun += a
            sky += b
        cnt = r.counters()
    assert cnt["gave_up"] == 0
    for name, g in (("sun", sun), ("sky", sky)):
        A = z[name + "_a"].astype(np.float64) / spp_ref
        B = z[name + "_b"].astype(np.float64) / spp_ref
        G = g / spp_g
        ok = np.isfinite(A).all(-1) & np.isfinite(B).all(-1)
        A, B, G = A[ok], B[ok], G[ok]
        for c in (slice(0, 3), slice(3, 4)):
            a, b, gg = A[:, c], B[:, c], G[:, c]
            noise2 = ((a - b) ** 2).sum() / 2.0 * (1.0 + spp_ref / spp_g)
            for x in (a, b):
                bias2 = ((gg - x) ** 2).sum() - noise2
                rel_bias = np.sqrt(max(bias2, 0.0) / (x ** 2).sum())
                assert rel_bias <= 0.01, (name, c, rel_bias, _rel(gg, x), _rel(a, b))
            # converged comparison: 4x4 box-filtered images against the reference mean
            ref_mean = 0.5 * (a + b)
            assert _rel(gg, ref_mean) < 0.05 + 1.5 * _rel(a, b) / np.sqrt(2.0)


def test_transmittance_vs_fp64_quadrature(gpu_renderer, port):
    """Delta-tracking transmittance along fixed rays from outside the volume,
    2^31 samples per ray, within 1e-4 relative of exp(-sigma_t * tau_FP64)."""
    nodes, bricks, _ = golden_octree()
    S = port.scene(nodes, bricks)
    sigma_t = float(np.float32(c0_cfg(8, 8)["sigma_s"]) + np.float32(c0_cfg(8, 8)["sigma_a"]))
    # rays from outside the volume towards it, kept when 0.6 < T < 0.95 so that
    # 5 standard errors of 2^31 samples stay below 1e-4 relative
    rng = np.random.default_rng(31)
    ro, rd, t_ref = [], [], []
    while len(ro) < 4:
        o = rng.uniform(-1.5, 2.5, 3)
        if (np.abs(o - 0.5) < 0.6).all():
            continue
        d = (0.5 + rng.uniform(-0.25, 0.25, 3)) - o
        d /= np.linalg.norm(d)
        of, df = o.astype(np.float32), d.astype(np.float32)
        o64, d64 = of.astype(np.float64), df.astype(np.float64)
        tau = port.L.orc_optical_depth(C.byref(S), o64.ctypes.data, d64.ctypes.data, 1e30)
        t = np.exp(-sigma_t * tau)
        if 0.6 < t < 0.95:
            ro.append(of)
            rd.append(df)
            t_ref.append(t)
    nsamp = 1 << 31
    t_gpu = gpu_renderer.probe_transmittance(np.array(ro), np.array(rd), nsamp, seed=31)
    for i in range(4):
        assert abs(t_gpu[i] - t_ref[i]) / t_ref[i] <= 1e-4, (i, t_gpu[i], t_ref[i])


def test_banded_host_render_equals_restatement(port):
    """dr_render_tile with host buffers renders a tall tile in row bands on two
    streams with pipelined copies; the result is the restatement's (odd last
    row left at zero, as the reference renders 2x2 blocks)."""
    from droplet_b200.renderer import Renderer
    from droplet_b200.scene import Octree

    nodes, bricks, mlevel = golden_octree()
    cfg = c0_cfg(40, 601)
    keep = []
    P = port.params(cfg, keep)
    S = port.scene(nodes, bricks)
    psun, psky, pcnt = port.render_tile(S, P, 0, 0, 40, 601, 8, seed=77, sample_base=16)
    with Renderer(0) as r:
        r.upload(Octree(nodes, bricks, mlevel))
        r.set_params(settings_from_cfg(cfg))
        for tuning in ((0, 5, 24, 0, 8), (0, 8, 24, 2, 0), (1, 0, 0, 0, 0)):
            r.set_tuning(*tuning)
            r.reset_counters()
            sun, sky = r.render_tile(0, 0, 40, 601, 8, seed=77, sample_base=16)
            cnt = r.counters()
            assert not sun[600].any() and not sky[600].any()
            for g, p in ((sun, psun), (sky, psky)):
                assert np.allclose(g, p, rtol=2e-5, atol=1e-6 * np.abs(p).max() + 1e-30), tuning
            for k in ("vertices", "density_lookups", "mie_evals", "paths"):
                assert cnt[k] == pcnt[k], (tuning, k)


def test_blocking_render_with_copy_threads_equals_device_render():
    """A tile whose row bands pass the 4 MB floor of the host copy threads
    (2048 x 512 pixels: 8 bands of 4.2 MB) comes back through the threaded
    copies equal to the same render into device buffers (the same paths; the
    per-pixel sums may differ in the order of their float additions)."""
    import torch

    from droplet_b200.renderer import Renderer
    from droplet_b200.scene import Octree

    nodes, bricks, mlevel = golden_octree()
    cfg = c0_cfg(2048, 512)
    with Renderer(0) as r:
        r.upload(Octree(nodes, bricks, mlevel))
        r.set_params(settings_from_cfg(cfg))
        r.set_tuning(0, 8, 24, 2, 0, 3, 1)
        for k in range(2):  # the second call reuses the started threads
            sun, sky = r.render_tile(0, 0, 2048, 512, 2, seed=5, sample_base=2 * k)
            dsun = torch.full((512, 2048, 4), -1.0, device="cuda")
            dsky = torch.full_like(dsun, -1.0)
            torch.cuda.synchronize()
            r.render_tile_async(0, 0, 2048, 512, 2, 5, 2 * k, dsun.data_ptr(), dsky.data_ptr())
            r.synchronize()
            for g, d in ((sun, dsun.cpu().numpy()), (sky, dsky.cpu().numpy())):
                assert np.isfinite(g).all() and g[..., 3].sum() > 0
                assert np.allclose(g, d, rtol=2e-5, atol=1e-6 * np.abs(d).max() + 1e-30), k


def test_large_sparse_scene_recipe_paths_equal_restatement(port):
    """The large sparse scene's recipe (24 puffs in a slab, sigma_t 100, 128
    events) at 256^3: GPU paths equal the restatement's."""
    from droplet_b200 import camera as cam
    from droplet_b200 import workloads as W
    from droplet_b200.renderer import Renderer
    from droplet_b200.scene import build_octree

    rec = W.slab_recipe(256)
    org, vals = W.sparse_field_puffwise(rec, device="cpu")
    oc = build_octree(org, vals, rec.voxel_size, 12)
    cfg = c0_cfg(160, 90)
    ss, sa, ev = W.medium("c4")
    cfg.update(sigma_s=ss, sigma_a=sa, scattevs=ev)
    eye = cam.orbit_eye(W.CENTER, W.CAMERA["distance"], W.CAMERA["azimuth"], 25.0)
    cfg["viewi"], cfg["proji"] = cam.camera_matrices(eye, W.CENTER, W.CAMERA["fov"], 160, 90)
    keep = []
    P = port.params(cfg, keep)
    S = port.scene(oc.nodes, oc.bricks)
    psun, psky, pcnt = port.render_tile(S, P, 40, 20, 80, 50, 16, seed=4, sample_base=0)
    assert pcnt["mie_evals"] > 3000  # the tile sees the puffs: paths scatter
    with Renderer(0) as r:
        r.upload(oc)
        r.set_params(settings_from_cfg(cfg))
        for tuning in ((0, 6, 20, 0, 0), (0, 8, 24, 2, 0, 3, 2), (1, 0, 0, 0, 0)):
            r.set_tuning(*tuning)
            r.reset_counters()
            sun, sky = r.render_tile(40, 20, 80, 50, 16, seed=4, sample_base=0)
            cnt = r.counters()
            for g, p in ((sun, psun), (sky, psky)):
                assert np.allclose(g, p, rtol=2e-5, atol=1e-6 * np.abs(p).max() + 1e-30), tuning
            for k in ("vertices", "density_lookups", "mie_evals", "paths"):
                assert cnt[k] == pcnt[k], (tuning, k)
