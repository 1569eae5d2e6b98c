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
    voxels of largest gradient (relative 1e-4);
  * the restatement's path-replay adjoint (the GPU adjoint's arithmetic, path
    for path) against it: see adjoint_vs_quadrature.

How the comparison reads.  The adjoint differentiates the probability of each
delta-tracking decision: w/rho for a real collision, -w/(rho_max - rho) for a
null one (w the voxel's trilinear weight).  Where the density is near zero a
real collision is rare and its weight 1/rho is huge, so the estimate is
unbiased but heavy-tailed: a finite sample misses the rare large terms.  So
the per-voxel check (2% plus 4 standard errors) takes the voxels of largest
gradient among those holding at least 1% of their leaf's majorant (2% plus 4
standard errors each, 1% in projection), and the projection onto the FP64
gradient over the largest-gradient voxels of all, near-empty ones included, is
held to 5%."""
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


def adjoint_vs_quadrature(g64, G, bricks, nodes):
    """(projection of the mean adjoint on the FP64 gradient over its 256
    largest entries, per-voxel failures among the 256 largest entries of voxels
    holding >= 1% of their leaf majorant, projection on those, median relative
    standard error there).  G: (groups, n_leaves * 512) independent estimates."""
    groups = G.shape[0]
    maj = np.zeros(len(bricks))
    fog = nodes["volx"][:, 1] != 0xFFFFFFFF
    maj[nodes["volx"][fog, 1]] = nodes["qval"][fog, 1]
    val = np.asarray(bricks, np.float64).ravel()
    gflat = g64.ravel()
    top = np.argsort(-np.abs(gflat))[:256]
    m_all = G[:, top].mean(0)
    proj_all = float(m_all @ gflat[top] / (gflat[top] @ gflat[top]))
    cand = np.flatnonzero(val >= 0.01 * np.repeat(maj, 512))
    sel = cand[np.argsort(-np.abs(gflat[cand]))[:256]]
    want = gflat[sel]
    m, se = G[:, sel].mean(0), G[:, sel].std(0, ddof=1) / np.sqrt(groups)
    bad = int((np.abs(m - want) > 0.02 * np.abs(want) + 4 * se).sum())
    return proj_all, bad, float(m @ want / (want @ want)), float(np.median(se / np.abs(want)))


def test_restated_adjoint_matches_quadrature_gradient(port):
    nodes, bricks, cfg, P, keep, ro, rd = crop_setup(port)
    S = port.scene(nodes, bricks)
    _, g64 = port.single_scatter_sun(S, P, ro, rd)
    spp, groups = 4096, 16
    dsun = np.zeros((16, 16, 4), np.float32)
    dsun[..., :3] = 1.0 / spp
    G = np.stack([np.asarray(port.adjoint_tile(S, P, 24, 24, 16, 16, spp, 700 + k, 0, dsun, np.zeros_like(dsun))[0],
                             np.float64).ravel() for k in range(groups)])
    proj_all, bad, proj, rel_se = adjoint_vs_quadrature(g64, G, bricks, nodes)
    assert abs(proj_all - 1.0) < 0.05, proj_all  # the near-empty voxels' heavy tails move it by a few %
    assert bad == 0 and abs(proj - 1.0) < 0.01, (bad, proj)
    assert rel_se < 0.04  # the check resolves a few per cent per voxel
