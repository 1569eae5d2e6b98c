"""Exact-mode Mie sampler (DR_PHASE_MIE_EXACT) on the GPU: the same samples as
the CPU restatement (whose distribution passes the chi-square test against the
tabulated phase function in test_oracle_pins), and exact-mode paths equal to
the restatement's."""
import numpy as np
import pytest

from conftest import c0_cfg, golden_octree, mie_table, settings_from_cfg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def exact_renderer():
    from droplet_b200.renderer import Renderer
    from droplet_b200.scene import Octree

    nodes, bricks, mlevel = golden_octree()
    r = Renderer(0)
    r.upload(Octree(nodes, bricks, mlevel))
    cfg = c0_cfg(64, 64)
    cfg["phase_mode"] = 1
    r.set_params(settings_from_cfg(cfg))
    yield r
    r.close()


def test_exact_sampler_equals_restatement(exact_renderer, port):
    from droplet_b200 import _native as N
    from scipy.stats import chi2

    import test_oracle_pins as T

    pdf, _ = mie_table()
    n = len(pdf)
    rng = np.random.default_rng(99)
    u = np.concatenate([rng.random(1_000_000, dtype=np.float32), np.linspace(0, 1, 4097, dtype=np.float32)[:-1]])
    got = exact_renderer.probe_sampler(N.DR_PROBE_MIE_EXACT_DIR, u, len(u))
    ct, st = port.mie_exact_dirs(port.mie_exact_table(pdf), n, u)
    assert np.array_equal(got[:, 0].view(np.uint32), ct.view(np.uint32))
    assert np.array_equal(got[:, 1].view(np.uint32), st.view(np.uint32))
    edges = np.linspace(0.0, np.pi, n + 1)
    counts = np.histogram(got[:1_000_000, 0].astype(np.float64), bins=-np.cos(edges))[0]
    m = T._phase_bin_masses(pdf[:, 0].astype(np.float64), edges)
    x2, dof = T._chi_square(counts, m / m.sum() * 1_000_000)
    assert chi2.sf(x2, dof) > 1e-4, (x2, dof)


@pytest.mark.parametrize("tuning", [(1, 0, 0, 0), (0, 5, 24, 0), (0, 8, 16, 1)])
def test_exact_mode_paths_equal_restatement(exact_renderer, port, tuning):
    nodes, bricks, _ = golden_octree()
    cfg = c0_cfg(64, 64)
    cfg["phase_mode"] = 1
    keep = []
    P = port.params(cfg, keep)
    S = port.scene(nodes, bricks)
    psun, psky, pcnt = port.render_tile(S, P, 8, 10, 48, 44, 48, seed=5, sample_base=0)
    saved = exact_renderer.get_tuning()
    try:
        exact_renderer.set_tuning(*tuning)
        exact_renderer.reset_counters()
        sun, sky = exact_renderer.render_tile(8, 10, 48, 44, 48, seed=5, sample_base=0)
        cnt = exact_renderer.counters()
    finally:
        exact_renderer.set_tuning(*saved)
    for g, p in ((sun, psun), (sky, psky)):
        assert np.allclose(g, p, rtol=2e-5, atol=1e-6 * np.abs(p).max() + 1e-30)
    for k in ("vertices", "density_lookups", "mie_evals", "paths"):
        assert cnt[k] == pcnt[k], (k, cnt[k], pcnt[k])
