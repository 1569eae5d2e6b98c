"""The FP64 single-scatter sun image (oracle/port/fp64.c,
orc_single_scatter_sun): the adjoint's independent check.  With one
scattering event the estimator's expected sun sum per path sample is a
deterministic integral along the camera ray (collision density times the
sun-cone average of phase-weighted shadow transmittance), computed by
Gauss-Legendre quadrature; its brick gradient is that quadrature's exact
derivative and shares no algebra with the path-replay adjoint (no
likelihood-ratio weights, no replay).

CPU checks (the GPU adjoint is compared against it in
tests/test_gpu_adjoint_fp64.py):
  * the quadrature equals the estimator (the restatement's Monte Carlo render
    of the same crop, 8 independent runs) within 4 standard errors and 0.2%;
  * its gradient equals central differences of the quadrature itself on the
    voxels of largest gradient (relative 1e-4)."""
import numpy as np
import pytest

from conftest import c0_cfg, golden_octree
from droplet_b200 import camera as cam


def crop_setup(port, x0=24, y0=24, n=16):
    nodes, bricks, _ = golden_octree()
    cfg = c0_cfg(64, 64)
    cfg["scattevs"] = 1
    keep = []
    P = port.params(cfg, keep)
    ys, xs = np.mgrid[y0:y0 + n, x0:x0 + n]
    ro, rd, inside = cam.camera_rays(cfg["viewi"], cfg["proji"], 64, 64, xs.ravel(), ys.ravel())
    assert inside.all()
    return nodes, bricks, cfg, P, keep, ro, rd


def test_quadrature_equals_the_estimator(port):
    nodes, bricks, cfg, P, keep, ro, rd = crop_setup(port, 28, 28, 8)
    S = port.scene(nodes, bricks)
    out, _ = port.single_scatter_sun(S, P, ro, rd, grad=False)
    want = out.sum(0)
    spp = 2048
    runs = np.array([port.render_tile(S, P, 28, 28, 8, 8, spp, seed=300 + k)[0][..., :3].sum((0, 1)) / spp
                     for k in range(8)])
    m, se = runs.mean(0), runs.std(0, ddof=1) / np.sqrt(len(runs))
    assert (want > 0).all()
    assert (np.abs(m - want) < 4 * se + 2e-3 * want).all(), (m, want, se)
    assert (se < 2e-3 * want).all()  # the check has the resolution it claims


def test_quadrature_gradient_equals_its_central_differences(port):
    nodes, bricks, cfg, P, keep, ro, rd = crop_setup(port, 28, 28, 4)
    S = port.scene(nodes, bricks)
    p_hit = port.sun_hit_fraction(P)
    _, g = port.single_scatter_sun(S, P, ro, rd, p_hit=p_hit)
    flat = np.argsort(-np.abs(g).ravel())[:6]
    b = np.array(bricks, np.float32)
    for idx in flat:
        li, vi = np.unravel_index(idx, g.shape)
        v0 = b[li, vi]
        vals = []
        steps = []
        for sgn in (1, -1):
            b[li, vi] = np.float32(v0 + sgn * 2.0 ** -9)
            steps.append(float(b[li, vi]))
            Sx = port.scene(nodes, b)
            vals.append(port.single_scatter_sun(Sx, P, ro, rd, grad=False, p_hit=p_hit)[0].sum())
        b[li, vi] = v0
        fd = (vals[0] - vals[1]) / (steps[0] - steps[1])
        assert abs(fd - g[li, vi]) <= 1e-4 * abs(g[li, vi]) + 1e-12, (idx, fd, g[li, vi])
