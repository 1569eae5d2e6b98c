"""Give-up reporting.  The reference has no iteration budgets: every path runs
to its end.  Here a path segment stops after a step budget of null collisions
(2^24 by default) and a block stops if its table staging times out, so a
result can be incomplete; the calls must say so instead of returning success.

The budget is set tiny (dr_set_step_budget), so that segments crossing the
config-0 cloud deterministically give up: a bounded loop that returns, not a
fault.  Checked: the blocking calls return DR_ERR_GAVE_UP (DrGaveUp) with the
tiles written and the counter raised; the asynchronous calls report through
dr_check_complete; a report is not repeated; the default budget reports
nothing; the libdroplet module raises from QueryResult."""
import time
from types import SimpleNamespace as NS

import numpy as np
import pytest

from conftest import c0_cfg, golden_octree, settings_from_cfg

pytestmark = pytest.mark.gpu


def _renderer():
    from droplet_b200.renderer import Renderer
    from droplet_b200.scene import Octree

    nodes, bricks, mlevel = golden_octree()
    r = Renderer(0)
    r.upload(Octree(nodes, bricks, mlevel))
    r.set_params(settings_from_cfg(c0_cfg(64, 64)))
    return r


def test_blocking_render_reports_give_ups():
    from droplet_b200 import _native as N

    with _renderer() as r:
        full_sun, full_sky = r.render_tile(16, 16, 32, 32, 8, seed=4, sample_base=0)
        assert r.counters()["gave_up"] == 0
        r.check_complete()  # nothing to report
        for kernel in (0, 1):  # persistent and per-path kernels
            r.set_tuning(kernel=kernel)
            r.set_step_budget(1)
            r.reset_counters()
            with pytest.raises(N.DrGaveUp, match="gave up") as ei:
                r.render_tile(16, 16, 32, 32, 8, seed=4, sample_base=0)
            assert ei.value.code == N.DR_ERR_GAVE_UP
            n = r.counters()["gave_up"]
            assert n > 0
            sun, sky = ei.value.result
            assert sun.shape == (32, 32, 4) and np.isfinite(sun).all()
            assert not np.allclose(sun, full_sun)  # the cut paths changed the tile
            # already reported by the blocking call: no second report
            r.check_complete()
            assert r.counters()["gave_up"] == n
            r.set_step_budget(0)
        r.set_tuning()
        sun, sky = r.render_tile(16, 16, 32, 32, 8, seed=4, sample_base=0)
        assert np.array_equal(sun, full_sun) or np.allclose(sun, full_sun, rtol=1e-5, atol=1e-6)


def test_blocking_shadow_reports_give_ups():
    from conftest import depth_texture
    from droplet_b200 import _native as N

    from droplet_b200.renderer import Renderer
    from droplet_b200.scene import Octree

    nodes, bricks, mlevel = golden_octree()
    with Renderer(0) as r:
        r.upload(Octree(nodes, bricks, mlevel))
        cfg = c0_cfg(64, 64)
        cfg["depth"] = depth_texture(64, 64)
        r.set_params(settings_from_cfg(cfg))
        r.render_shadow_tile(0, 0, 64, 64, 4, seed=2, sample_base=0)
        r.set_step_budget(1)
        with pytest.raises(N.DrGaveUp):
            r.render_shadow_tile(0, 0, 64, 64, 4, seed=2, sample_base=0)


def test_async_calls_report_through_check_complete():
    import torch

    from droplet_b200 import _native as N
    from droplet_b200.renderer import stream_handle

    with _renderer() as r:
        sun = torch.zeros((32, 32, 4), device="cuda")
        sky = torch.zeros_like(sun)
        st = torch.cuda.current_stream()
        h = stream_handle(st)
        r.render_tile_async(16, 16, 32, 32, 8, 4, 0, sun.data_ptr(), sky.data_ptr(), h)
        r.check_complete(h)
        r.set_step_budget(1)
        r.set_params(settings_from_cfg(c0_cfg(64, 64)))  # the budget survives new parameters
        r.render_tile_async(16, 16, 32, 32, 8, 4, 0, sun.data_ptr(), sky.data_ptr(), h)
        with pytest.raises(N.DrGaveUp, match="since the last check"):
            r.check_complete(h)
        r.check_complete(h)  # reported once
        r.set_step_budget(0)
        r.render_tile_async(16, 16, 32, 32, 8, 4, 0, sun.data_ptr(), sky.data_ptr(), h)
        r.check_complete(h)


def test_batch_reports_through_check_complete():
    from droplet_b200 import _native as N
    from droplet_b200.renderer import Batch, BatchView
    from droplet_b200.scene import Octree

    nodes, bricks, mlevel = golden_octree()
    with _renderer() as r:
        s = settings_from_cfg(c0_cfg(64, 64))
        oc = Octree(nodes, bricks, mlevel)
        r.set_step_budget(1)
        b = Batch(r, [oc], [BatchView(0, s, 4, 1)])
        try:
            b.launch()
            with pytest.raises(N.DrGaveUp):
                r.check_complete()
        finally:
            b.close()


def test_libdroplet_query_result_raises_after_a_give_up():
    import importlib

    import libdroplet
    from conftest import mie_table, sky_state_c0
    from test_libdroplet import fake_scene

    lib = importlib.reload(libdroplet)
    pdf, cdf = mie_table()
    lib.SetPhaseTable(pdf, cdf)
    lib.SetSkyState(*sky_state_c0())
    try:
        lib.BeginRender(fake_scene(), NS(), 32, 32, 64, 64, 1)
        t = time.time()
        while lib.QueryStatus() != 0:
            assert time.time() - t < 60
            time.sleep(0.01)
        lib._renderer.set_step_budget(1)
        lib.Render(16, 16, 32, 32, 8)
        t = time.time()
        while lib.QueryStatus() != 0:
            assert time.time() - t < 60
            time.sleep(0.01)
        with pytest.raises(SystemError, match="gave up"):
            lib.QueryResult(0)
        lib._renderer.set_step_budget(0)
        lib.Render(16, 16, 32, 32, 8)
        while lib.QueryResult(0) is None:
            time.sleep(0.01)
        assert len(lib.QueryResult(1)) == 32 * 32
    finally:
        lib.EndRender()
