"""The GPU path-replay adjoint against the FP64 single-scatter quadrature
gradient (oracle/port/fp64.c; checked there against the estimator and its own
central differences by tests/test_single_scatter_fp64.py).  This check shares
no likelihood-ratio algebra with the adjoint.

Config 0 with one scattering event, a 16x16 crop of the 64x64 frame, loss
L = sum over pixels and rgb of the sun sums per sample (dsun = 1/spp, dsky = 0).
The adjoint runs 16 independent seed groups of 16384 spp (67 M paths).  The
criteria are those of tests/test_single_scatter_fp64.py (where the reason for
the density threshold is given): the projection of the mean adjoint on the FP64
gradient's 256 largest entries within 5% (0.969 on the GPU at 16 x 16384 spp, 1.003 with the
restatement at 16 x 4096 spp: the near-empty voxels among them have
heavy-tailed estimates); among voxels holding at least 1% of
their leaf majorant, the 256 of largest gradient each within 2% plus 4 standard
errors and their projection within 1%."""
import numpy as np
import pytest

from conftest import settings_from_cfg
from test_single_scatter_fp64 import adjoint_vs_quadrature, crop_setup

pytestmark = pytest.mark.gpu


def test_adjoint_matches_fp64_single_scatter_gradient(port):
    import torch

    from droplet_b200.renderer import Renderer
    from droplet_b200.scene import Octree
    from conftest import golden_octree

    nodes, bricks, cfg, P, keep, ro, rd = crop_setup(port)
    S = port.scene(nodes, bricks)
    out, g64 = port.single_scatter_sun(S, P, ro, rd)
    spp, groups = 16384, 16
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
    proj_all, bad, proj, rel_se = adjoint_vs_quadrature(g64, G.reshape(groups, -1), bricks, nodes)
    assert abs(proj_all - 1.0) < 0.05, proj_all  # the near-empty voxels' heavy tails move it by a few %
    assert bad == 0 and abs(proj - 1.0) < 0.01, (bad, proj)
    assert rel_se < 0.02, rel_se  # the check resolves 2% per voxel
