"""The path-replay adjoint restated on the CPU (oracle/port), pinned without a
GPU: the FP64 quadrature gradient of the optical depth against its own finite
differences, the delta-tracking transmittance adjoint against that FP64
gradient, and the image adjoint's albedo derivative against central finite
differences with common random numbers (albedo changes no tracking decision,
so the CRN difference quotient is the derivative of the same paths)."""
import numpy as np
import pytest

from conftest import c0_cfg, golden_octree


def _rays(nodes, n, seed):
    rng = np.random.default_rng(seed)
    ro = np.zeros((n, 3))
    rd = np.zeros((n, 3))
    for i in range(n):
        # from outside the cube towards a point near the centre
        o = np.array([0.5, 0.5, 0.5]) + 2.0 * rng.normal(size=3) / np.sqrt(3)
        t = np.array([0.5, 0.5, 0.5]) + rng.uniform(-0.15, 0.15, 3)
        d = t - o
        ro[i], rd[i] = o, d / np.linalg.norm(d)
    return ro, rd


def test_fp64_optical_depth_gradient_matches_finite_differences(port):
    nodes, bricks, _ = golden_octree()
    ro, rd = _rays(nodes, 3, 1)
    b = np.array(bricks, np.float32, copy=True)
    S = port.scene(nodes, b)
    for i in range(3):
        g = port.optical_depth_grad(S, ro[i], rd[i])
        nz = np.argwhere(g.reshape(-1) != 0).ravel()
        assert len(nz) > 50
        pick = np.random.default_rng(i).choice(nz, 12, replace=False)
        for k in pick:
            h = 1e-3
            flat = b.reshape(-1)
            v0 = flat[k]
            flat[k] = v0 + h
            tp = port.optical_depth(S, ro[i], rd[i])
            flat[k] = v0 - h
            tm = port.optical_depth(S, ro[i], rd[i])
            flat[k] = v0
            fd = (tp - tm) / (np.float64(np.float32(v0 + h)) - np.float64(np.float32(v0 - h)))
            assert abs(fd - g.reshape(-1)[k]) <= 1e-6 + 1e-5 * abs(fd), (i, k, fd, g.reshape(-1)[k])


def test_transmittance_adjoint_matches_fp64_gradient(port):
    """Score-function gradient of the delta-tracking transmittance (escaped
    samples replay their null decisions) against -sigma_t T dtau/dv in FP64."""
    nodes, bricks, _ = golden_octree()
    cfg = c0_cfg(8, 8)
    keep = []
    P = port.params(cfg, keep)
    S = port.scene(nodes, bricks)
    st = cfg["sigma_s"] + cfg["sigma_a"]
    ro, rd = _rays(nodes, 4, 2)
    for i in range(4):
        g_mc, T = port.adjoint_transmittance(S, P, ro[i:i + 1].astype(np.float32), rd[i:i + 1].astype(np.float32),
                                             np.ones(1, np.float32), 200000, 11 + i)
        tau = port.optical_depth(S, ro[i], rd[i])
        Tref = np.exp(-st * tau)
        g_ref = -st * Tref * port.optical_depth_grad(S, ro[i], rd[i])
        assert abs(T[0] - Tref) < 4 * np.sqrt(Tref * (1 - Tref) / 200000) + 1e-4
        a, r = g_mc.ravel(), g_ref.ravel()
        proj = float(a @ r / (r @ r))
        assert abs(proj - 1.0) < 0.03, (i, proj)
        assert np.linalg.norm(a - r) / np.linalg.norm(r) < 0.25, i


def test_albedo_adjoint_matches_crn_finite_differences(port):
    nodes, bricks, _ = golden_octree()
    w = h = 24
    cfg = c0_cfg(w, h)
    st = cfg["sigma_s"] + cfg["sigma_a"]
    S = port.scene(nodes, bricks)
    rng = np.random.default_rng(3)
    dsun = rng.normal(size=(h, w, 4)).astype(np.float32)
    dsky = rng.normal(size=(h, w, 4)).astype(np.float32)

    def loss(albedo):
        c = dict(cfg)
        c["sigma_s"] = float(np.float32(st * albedo))
        c["sigma_a"] = float(np.float32(st) - np.float32(st * albedo))
        keep = []
        P = port.params(c, keep)
        sun, sky, _ = port.render_tile(S, P, 0, 0, w, h, 64, seed=5)
        return float((dsun[..., :3].astype(np.float64) * sun[..., :3]).sum()
                     + (dsky[..., :3].astype(np.float64) * sky[..., :3]).sum()), P, keep

    a0 = 0.99
    _, P0, keep0 = loss(a0)
    f0 = float(np.float32(np.float32(st * a0) / (np.float32(st - np.float32(st * a0)) + np.float32(st * a0))))
    _, galb = port.adjoint_tile(S, P0, 0, 0, w, h, 64, 5, 0, dsun, dsky)
    eps = 1e-3
    lp, _, _ = loss(a0 + eps)
    lm, _, _ = loss(a0 - eps)
    fd = (lp - lm) / (2 * eps)
    assert abs(galb - fd) < 0.02 * abs(fd) + 1e-6, (galb, fd, f0)


def test_sky_zero_over_zero_path_and_finite_paths_flag(port):
    """The reference's sky term divides rd.x by rd.y (src/kernel.cpp:338-342):
    a path escaping along a direction with rd.y == 0 sums to NaN.  The CPU
    restatement reproduces it; DR_KERNEL_FINITE_PATHS drops such a sample."""
    from conftest import NAN_PATH, orbit_cfg, uniform_cube_scene

    nodes, bricks, _ = uniform_cube_scene(port.build_octree)
    S = port.scene(nodes, bricks)
    cfg = orbit_cfg(256, 256, 0.0)
    keep = []
    P = port.params(cfg, keep)
    px, py = NAN_PATH["pixel"]
    sun, sky, _ = port.render_path(S, P, px, py, NAN_PATH["seed"], NAN_PATH["sample"])
    assert np.isnan(sky[:3]).all() and np.isfinite(sun).all()
    cfg["finite_paths"] = True
    P = port.params(cfg, keep)
    sun, sky, _ = port.render_path(S, P, px, py, NAN_PATH["seed"], NAN_PATH["sample"])
    assert (sky[:3] == 0).all() and (sun[:3] == 0).all() and sun[3] == 1.0


def test_density_adjoint_matches_reweighted_finite_differences(port):
    """The image adjoint's brick-sample derivative equals central differences of
    the reweighted replay (decisions from the base bricks, each weighted by its
    probability ratio under the perturbed bricks) on the same random streams;
    with unperturbed bricks the reweighted loss is the plain render's."""
    nodes, bricks, _ = golden_octree()
    w = h = 24
    spp = 16
    cfg = c0_cfg(w, h)
    S = port.scene(nodes, bricks)
    keep = []
    P = port.params(cfg, keep)
    rng = np.random.default_rng(11)
    dsun = rng.normal(size=(h, w, 4)).astype(np.float32)
    dsky = rng.normal(size=(h, w, 4)).astype(np.float32)
    base = np.asarray(bricks, np.float32).reshape(-1, 512)
    sun, sky, _ = port.render_tile(S, P, 0, 0, w, h, spp, seed=5)
    plain = float((dsun[..., :3].astype(np.float64) * sun[..., :3]).sum()
                  + (dsky[..., :3].astype(np.float64) * sky[..., :3]).sum())
    l0 = port.reweighted_loss(S, P, 0, 0, w, h, spp, 5, 0, dsun, dsky, base)
    assert abs(l0 - plain) <= 1e-5 * abs(plain)
    g, _ = port.adjoint_tile(S, P, 0, 0, w, h, spp, 5, 0, dsun, dsky)
    flat = base.reshape(-1)
    cand = np.flatnonzero(flat >= 0.05)
    pick = rng.choice(cand, 256, replace=False)
    u = np.zeros(flat.size, np.float32)
    u[pick] = rng.choice([-1.0, 1.0], 256)
    u = u.reshape(base.shape)
    eps = 1e-3
    lp = port.reweighted_loss(S, P, 0, 0, w, h, spp, 5, 0, dsun, dsky, base + eps * u)
    lm = port.reweighted_loss(S, P, 0, 0, w, h, spp, 5, 0, dsun, dsky, base - eps * u)
    fd = (lp - lm) / (2 * eps)
    ad = float((g * u).sum())
    assert abs(ad) > 0
    assert abs(fd - ad) <= 1e-3 * abs(ad), (fd, ad)
