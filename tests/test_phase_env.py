"""The Henyey-Greenstein phase (HGPhase, src/KernelSampler.cpp:164-204) and the
environment light of the reference's default build (NullEnv / MapEnv,
src/KernelSampler.cpp:355-417, src/kernel.cpp:361-364), restated in the CPU
oracle and pinned to the compiled reference: atan2 and MapEnv::Evaluate bit for
bit, HG within the ulps that powf and the restatement's pow differ by, and
rendered images statistically (16 independent runs a side)."""
import numpy as np
import pytest

from conftest import c0_cfg, golden_octree


def _dirs(n, seed):
    rng = np.random.default_rng(seed)
    rd = rng.normal(size=(n, 3))
    rd /= np.linalg.norm(rd, axis=1, keepdims=True)
    axes = np.array([[0, 0, 1], [0, 0, -1], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 0]], np.float64)
    return np.vstack([rd, axes]).astype(np.float32)


def env_map(seed=2, h=33, w=64):
    """An RGBA environment map with smooth structure and texel noise (seeded)."""
    rng = np.random.default_rng(seed)
    j, i = np.mgrid[0:h, 0:w]
    base = np.stack([0.6 + 0.4 * np.cos(np.pi * j / h), 0.5 + 0.3 * np.sin(2 * np.pi * i / w),
                     0.4 + 0.2 * (j / h), np.ones_like(j, np.float64)], -1)
    return (base * rng.uniform(0.8, 1.2, (h, w, 4))).astype(np.float32)


def test_atan2_bit_exact_vs_reference(port, ref):
    rng = np.random.default_rng(3)
    y = np.concatenate([rng.normal(size=20000), [0, 0, 1, -1, 0]]).astype(np.float32)
    x = np.concatenate([rng.normal(size=20000), [0, 1, 0, 0, -1]]).astype(np.float32)
    a, b = ref.atan2(y, x), port.atan2_ref(y, x)
    assert np.array_equal(np.isnan(a), np.isnan(b))
    assert np.array_equal(a[~np.isnan(a)].view(np.uint32), b[~np.isnan(b)].view(np.uint32))


def test_env_map_bit_exact_vs_reference(port, ref):
    """Including the reference's extrapolation past the last texel row for a
    ray straight up and the 0/0 of atan2 on the z axis."""
    em = env_map()
    rd = _dirs(20000, 4)
    cfg = c0_cfg(16, 16)
    cfg["env_mode"], cfg["env_map"] = 2, em
    keep = []
    P = port.params(cfg, keep)
    a, b = ref.env_eval(em, rd), port.env_map_eval(P, rd)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert (a[-7] < 0).any()  # (0, 0, 1): extrapolated beyond the map


@pytest.mark.parametrize("g", [0.75, -0.3, 0.2])
def test_hg_phase_vs_reference(port, ref, g):
    rng = np.random.default_rng(5)
    ct = rng.uniform(-1, 1, 20000).astype(np.float32)
    a, b = ref.hg_eval(g, ct), port.hg_eval(g, ct)
    assert np.max(np.abs(a - b) / np.abs(a)) < 2e-6  # powf vs the restatement's pow: a few ulps
    iv = _dirs(5000, 6)[:5000]
    u1 = rng.random(5000).astype(np.float32)
    u2 = rng.random(5000).astype(np.float32)
    a, b = ref.hg_sample(g, iv, u1, u2), port.hg_sample(g, iv, u1, u2)
    assert np.max(np.abs(a - b)) < 2e-6


def test_hg_samples_follow_the_hg_density(port):
    """Chi-square of cos(theta) of 2e5 HG samples against the HG density."""
    g = 0.75
    rng = np.random.default_rng(7)
    n = 200000
    iv = np.tile(np.array([[0.3, 0.4, 0.866]], np.float32), (n, 1))
    iv /= np.linalg.norm(iv, axis=1, keepdims=True)
    d = port.hg_sample(g, iv, rng.random(n).astype(np.float32), rng.random(n).astype(np.float32))
    ct = np.clip((d * iv).sum(1), -1, 1)
    edges = np.linspace(-1, 1, 41)
    obs, _ = np.histogram(ct, edges)

    def cdf(c):  # integral of 2 pi p(ct) dct, p the HG density
        return (1 - g * g) / (2 * g) * (1 / np.sqrt(1 + g * g - 2 * g * c) - 1 / (1 + g))

    exp = n * np.diff(cdf(edges))
    chi2 = ((obs - exp) ** 2 / exp).sum()
    assert chi2 < 80  # 39 dof: p ~ 1e-4


def _agree(R, Q, label, z=4.5):
    r, q = np.asarray(R, np.float64), np.asarray(Q, np.float64)
    assert np.isfinite(r).all() and np.isfinite(q).all(), label
    se = np.sqrt(r.var(ddof=1) / len(r) + q.var(ddof=1) / len(q)) + 1e-12 * abs(r.mean())
    assert abs(r.mean() - q.mean()) < z * se + 1e-9, (label, r.mean(), q.mean(), se)


RUNS = 16


@pytest.mark.parametrize("mode", ["hg", "envmap", "nullenv"])
def test_port_render_matches_reference_statistically(port, mode):
    """HG (the Hosek build) and the environment-map and null-environment
    builds: image sums of 16 independent runs a side agree within 4.5
    standard errors; without an environment no sky light reaches the image."""
    from oracle import Reference, ref_available
    from oracle.oracle import REF_ENV_LIB

    if not ref_available():
        pytest.skip("reference oracle not built")
    ref = Reference() if mode == "hg" else Reference(REF_ENV_LIB)
    nodes, bricks, _ = golden_octree()
    cfg = c0_cfg(16, 16)
    if mode == "hg":
        cfg["phase_mode"], cfg["hg_g"] = 2, 0.75
    else:
        cfg["env_mode"] = 2 if mode == "envmap" else 1
        if mode == "envmap":
            cfg["env_map"] = env_map()
    rs = ref.scene(nodes, bricks)
    ref.set_threads(0)
    keep = []
    P = port.params(cfg, keep)
    S = port.scene(nodes, bricks)
    spp = 512
    R = [rs.render_ex(cfg, 0, 0, 16, 16, spp) for _ in range(RUNS)]
    Q = [port.render_tile(S, P, 0, 0, 16, 16, spp, seed=2000 + k)[:2] for k in range(RUNS)]
    for bi in range(2):
        for ch in range(4):
            _agree([x[bi][..., ch].sum() / spp for x in R], [x[bi][..., ch].sum() / spp for x in Q], (mode, bi, ch))
    if mode == "nullenv":
        assert not any(x[1][..., :3].any() for x in R) and not any(x[1][..., :3].any() for x in Q)
