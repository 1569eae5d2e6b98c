"""Batched rendering (dr_batch_*): several scenes and views of uneven size in
one persistent launch replayed from a CUDA graph.  Every view of launch k
equals the CPU restatement's tile for sample_base = k spp (up to the order of
the per-pixel float sums), and the counters equal the sum over views."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, depth_texture, golden_octree, mie_table, settings_from_cfg
from droplet_b200 import camera as cam
from droplet_b200 import workloads as W

pytestmark = pytest.mark.gpu


def sky_for_degree(deg):
    with open(os.path.join(GOLDEN, "sky_states_by_degree.json")) as f:
        s = next(x for x in json.load(f) if x["degree"] == deg)
    return np.asarray(s["configs"]), np.asarray(s["radiances"])


def view_cfg(w, h, azimuth, sun_deg, sigma_t, scattevs):
    pdf, cdf = mie_table()
    cfgs, rads = sky_for_degree(sun_deg)
    eye = cam.orbit_eye(W.CENTER, W.CAMERA["distance"], azimuth, W.CAMERA["elevation"])
    viewi, proji = cam.camera_matrices(eye, W.CENTER, W.CAMERA["fov"], w, h)
    ss, sa, ev = W.medium_of(sigma_t, 0.99, scattevs)
    return dict(sigma_s=ss, sigma_a=sa, scattevs=ev, sun_dir=cam.sun_direction(sun_deg, W.SUN["azimuth"]),
                sun_color=np.asarray(W.SUN["color"], np.float32), sun_angle=W.SUN["angle"], sky_configs=cfgs,
                sky_radiances=rads, mie_pdf=pdf, mie_cdf=cdf, viewi=viewi, proji=proji, w=w, h=h)


@pytest.fixture(scope="module")
def batch_setup():
    from droplet_b200.renderer import Batch, BatchView, Renderer
    from droplet_b200.scene import Octree, build_octree

    nodes, bricks, mlevel = golden_octree()
    oc0 = Octree(nodes, bricks, mlevel)
    rec = W.config0_recipe(48, 12)
    org, vals = W.sparse_field(rec)
    oc1 = build_octree(org, vals, rec.voxel_size, 12)
    from test_phase_env import env_map

    c3 = view_cfg(64, 64, 200.0, 60, 30.0, 12)
    c3["depth"] = depth_texture(64, 64)
    c3["depthcomp"] = True
    c1 = view_cfg(96, 80, 35.0, 45, 45.0, 16)
    c1["env_mode"] = 1  # NullEnv
    c2 = view_cfg(40, 40, 120.0, 12, 70.0, 500)
    c2.update(phase_mode=2, hg_g=0.6, env_mode=2, env_map=env_map())  # HG phase, MapEnv
    specs = [  # (scene, cfg, region, spp, seed)
        (0, view_cfg(64, 64, -90.0, 30, 20.0, 8), None, 24, 3),
        (1, c1, (8, 4, 72, 60), 16, 4),
        (0, c2, None, 40, 5),
        (1, c3, (2, 2, 61, 59), 8, 6),
    ]
    r = Renderer(0)
    views = [BatchView(s, settings_from_cfg(c), spp, seed, reg) for s, c, reg, spp, seed in specs]
    b = Batch(r, [oc0, oc1], views)
    yield r, b, specs, [oc0, oc1]
    b.close()
    r.close()


def check_launches(r, b, specs, scenes, port, tag):
    """Two launches of b: every view equals the restatement's tile for
    sample_base = k spp, the counters equal the sum over views."""
    S = [port.scene(oc.nodes, oc.bricks) for oc in scenes]
    for _ in range(2):
        _, k = b.info()
        r.reset_counters()
        b.launch()
        got = [b.read(v) for v in range(len(specs))]
        cnt = r.counters()
        total = dict.fromkeys(("vertices", "density_lookups", "mie_evals", "paths"), 0)
        for v, (s, cfg, reg, spp, seed) in enumerate(specs):
            keep = []
            P = port.params(cfg, keep)
            x0, y0, tw, th = reg if reg is not None else (0, 0, cfg["w"], cfg["h"])
            psun, psky, pcnt = port.render_tile(S[s], P, x0, y0, tw, th, spp, seed=seed, sample_base=k * spp)
            for g, p in zip(got[v], (psun, psky)):
                assert g.shape == p.shape
                assert np.allclose(g, p, rtol=2e-5, atol=1e-6 * np.abs(p).max() + 1e-30), (v, tag)
            for key in total:
                total[key] += pcnt[key]
        for key, val in total.items():
            assert cnt[key] == val, (key, cnt[key], val, tag)
    n, launches = b.info()
    assert n > 0 and launches >= 2


@pytest.mark.parametrize("tuning", [(0, 5, 24, 0, 0), (0, 8, 16, 1, 8), (0, 4, 8, 0, 16), (0, 8, 24, 2, 0),
                                    (0, 6, 16, 2, 8)])
def test_batch_views_equal_restatement(batch_setup, port, tuning):
    r, b, specs, scenes = batch_setup
    b.set_tuning(*tuning)
    assert b.get_tuning()[1:5] == tuning[1:5]
    assert b.get_split()[1] == 0  # these views are far below the automatic split size
    check_launches(r, b, specs, scenes, port, tuning)


# split graphs: views of at least `split` paths run in plain persistent kernels
# of their own (independent graph branches, the launch counter read on the
# device), the rest in the batched kernel; 60,000 paths leaves the last view
# (60 x 58 pixels x 8 spp) to the batched kernel in both pixel orders
@pytest.mark.parametrize("split,own", [(1, 4), (60_000, 3), (0, 0)])
@pytest.mark.parametrize("tuning", [(0, 8, 24, 2, 0), (0, 5, 16, 1, 8), (0, 6, 8, 0, 16)])
def test_batch_split_views_equal_restatement(batch_setup, port, tuning, split, own):
    from droplet_b200.renderer import Batch

    r, b, specs, scenes = batch_setup
    b.set_tuning(*tuning)
    b.set_split(split)
    try:
        assert b.get_split() == (split, own)
        check_launches(r, b, specs, scenes, port, (tuning, split))
    finally:
        b.set_split(Batch.SPLIT_AUTO)


def test_batch_rejects_mixed_phase_tables(batch_setup):
    from droplet_b200 import _native as N
    from droplet_b200.renderer import Batch, BatchView

    r, _, specs, scenes = batch_setup
    c = dict(specs[0][1])
    c2 = dict(c)
    c2["phase_mode"] = 1
    with pytest.raises(N.DrError):
        Batch(r, scenes, [BatchView(0, settings_from_cfg(c), 4), BatchView(0, settings_from_cfg(c2), 4)])
