"""The GPU path-replay adjoint against the FP64 single-scatter quadrature
gradient (oracle/port/fp64.c; checked there against the estimator and its own
central differences by tests/test_single_scatter_fp64.py).  This check shares
no likelihood-ratio algebra with the adjoint.

Config 0 with one scattering event, a 16x16 crop of the 64x64 frame, loss
L = sum over pixels and rgb of the sun sums per sample (dsun = 1/spp, dsky = 0).
The adjoint runs 16 independent seed groups of 2048 spp (8.4 M paths); on the
256 voxels of largest FP64 gradient each voxel's mean agrees within 2% plus 4
standard errors, and the projection of the adjoint on the FP64 gradient is
within 1% of it."""
import numpy as np
import pytest

from conftest import settings_from_cfg
from test_single_scatter_fp64 import crop_setup

pytestmark = pytest.mark.gpu


def test_adjoint_matches_fp64_single_scatter_gradient(port):
    import torch

    from droplet_b200.renderer import Renderer
    from droplet_b200.scene import Octree
    from conftest import golden_octree

    nodes, bricks, cfg, P, keep, ro, rd = crop_setup(port)
    S = port.scene(nodes, bricks)
    out, g64 = port.single_scatter_sun(S, P, ro, rd)
    spp, groups = 2048, 16
    n = 16
    with Renderer(0) as r:
        _, _, mlevel = golden_octree()
        r.upload(Octree(nodes, bricks, mlevel))
        r.set_params(settings_from_cfg(cfg))
        ds = torch.zeros((n, n, 4), device="cuda")
        ds[..., :3] = 1.0 / spp
        dk = torch.zeros_like(ds)
        gs = []
        fw = []
        sun = torch.zeros((n, n, 4), device="cuda")
        sky = torch.zeros_like(sun)
        for k in range(groups):
            g = torch.zeros((len(bricks), 512), dtype=torch.float32, device="cuda")
            ga = torch.zeros(1, dtype=torch.float64, device="cuda")
            r.adjoint_tile_async(24, 24, n, n, spp, 700 + k, 0, ds.data_ptr(), dk.data_ptr(), g.data_ptr(),
                                 ga.data_ptr())
            r.render_tile_async(24, 24, n, n, spp, 900 + k, 0, sun.data_ptr(), sky.data_ptr(),
                                int(torch.cuda.current_stream().cuda_stream) or 1)
            torch.cuda.synchronize()
            gs.append(g.cpu().numpy().astype(np.float64))
            fw.append(sun[..., :3].sum().item() / spp)
        r.check_complete()
    G = np.stack(gs)
    # the forward image agrees with the quadrature (the model the gradient differentiates)
    fw = np.asarray(fw)
    assert abs(fw.mean() - out.sum()) < 4 * fw.std(ddof=1) / np.sqrt(groups) + 2e-3 * out.sum()
    top = np.argsort(-np.abs(g64).ravel())[:256]
    want = g64.ravel()[top]
    got = G.reshape(groups, -1)[:, top]
    m, se = got.mean(0), got.std(0, ddof=1) / np.sqrt(groups)
    bad = np.abs(m - want) > 0.02 * np.abs(want) + 4 * se
    assert bad.sum() == 0, (np.flatnonzero(bad)[:8], m[bad][:8], want[bad][:8], se[bad][:8])
    proj = float(m @ want / (want @ want))
    assert abs(proj - 1.0) < 0.01, proj
    assert float(np.median(se / np.abs(want))) < 0.02  # the check resolves 2%
