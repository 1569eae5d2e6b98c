"""Scenes, rays and crops of the deep-octree parity checks (the benchmark
configurations' octree depths, against the compiled reference).

  c1  the 512^3 cumulus (workloads.cumulus_recipe): depth 6; medium of the
      cumulus frame (sigma_t 60, albedo 0.999, 64 events); crop = the 32x32
      centre of its 1920x1080 frame.
  c4  puffs 15, 23, 6 and 12 of the large sparse scene (workloads.slab_recipe)
      on its 2048^3 grid: far apart, so the root box spans the slab and the
      octree has the large scene's depth 8; medium of the large scene (sigma_t
      100, albedo 0.99, 128 events); camera of its 3840x2160 frame, crop = the
      32x32 block centred on puff 15.
Used by tests/golden/make_golden_deep.py (which writes the reference's
fixtures) and by the tests that check the restatement and the GPU against them.
"""
from __future__ import annotations

import numpy as np

from droplet_b200 import camera as cam
from droplet_b200 import workloads as W

CONFIGS = {
    "c1": {"depth": 6, "medium": "c1", "rays": 3000, "ray_seed": 61},
    "c4": {"depth": 8, "medium": "c4", "rays": 3000, "ray_seed": 84},
}
C4_PUFFS = (15, 23, 6, 12)


def recipe(name: str) -> W.FieldRecipe:
    if name == "c1":
        return W.cumulus_recipe(512)
    rec = W.slab_recipe(2048)
    return W.FieldRecipe(rec.n, [rec.puffs[i] for i in C4_PUFFS], extent=rec.extent)


def build_field(name: str, device: str = "cpu"):
    """(block origins, block values, recipe) of the configuration's field; the
    same generator on every device (float64 operations that round alike)."""
    rec = recipe(name)
    if name == "c1":
        org = W.candidate_blocks(rec)
        vals = W.eval_blocks_torch(rec, org, device=device)
        nz = (vals != 0).any(1)
        return np.ascontiguousarray(org[nz]), np.ascontiguousarray(vals[nz]), rec
    org, vals = W.sparse_field_puffwise(rec, device=device)
    return org, vals, rec


def ray_set(nodes, n: int, seed: int):
    """n rays through the octree: a third from outside the root box aimed at
    points inside it, a third from outside aimed at random leaves, a third
    starting inside random leaves in random directions; every 50th ray is
    axis-parallel (the traversal's NaN-midpoint case)."""
    rng = np.random.default_rng(seed)
    ce = np.asarray(nodes["ce"][0], np.float64)
    c, e = ce[:3], float(ce[3])
    leaves = np.nonzero(nodes["volx"][:, 1] != 0xFFFFFFFF)[0]
    lc = np.asarray(nodes["ce"][rng.choice(leaves, n)], np.float64)
    pin = lc[:, :3] + rng.uniform(-0.9, 0.9, (n, 3)) * lc[:, 3:4]  # points inside random leaves
    out = c + rng.uniform(-2.5, 2.5, (n, 3)) * e
    out += np.sign(out - c) * e  # outside the root box
    k1, k2 = n // 3, 2 * n // 3
    ro = np.empty((n, 3))
    rd = np.empty((n, 3))
    ro[:k1] = out[:k1]
    rd[:k1] = (c + rng.uniform(-0.8, 0.8, (k1, 3)) * e) - ro[:k1]
    ro[k1:k2] = out[k1:k2]
    rd[k1:k2] = pin[k1:k2] - ro[k1:k2]
    ro[k2:] = pin[k2:]
    rd[k2:] = rng.normal(size=(n - k2, 3))
    for i in range(0, n, 50):
        rd[i] = 0.0
        rd[i, (i // 50) % 3] = 1.0 if (i // 50) % 2 else -1.0
    rd /= np.linalg.norm(rd, axis=1, keepdims=True)
    return ro.astype(np.float32), rd.astype(np.float32)


def _frame(name: str):
    if name == "c1":
        eye = cam.orbit_eye(W.CENTER, W.CAMERA["distance"], W.CAMERA["azimuth"], W.CAMERA["elevation"])
        return eye, 1920, 1080
    eye = cam.orbit_eye(W.CENTER, W.CAMERA["distance"], W.CAMERA["azimuth"], 25.0)
    return eye, 3840, 2160


def crop_origin(name: str, viewi, proji, w: int, h: int):
    """Top-left pixel (even) of the 32x32 crop."""
    if name == "c1":
        return w // 2 - 16, h // 2 - 16
    p = np.asarray(W.slab_recipe(2048).puffs[15].center, np.float64)
    ys, xs = np.mgrid[0:h:4, 0:w:4]
    ro, rd, _ = cam.camera_rays(viewi, proji, w, h, xs.ravel(), ys.ravel())
    v = p - ro.astype(np.float64)
    d = rd.astype(np.float64)
    dist = np.linalg.norm(v - (v * d).sum(1, keepdims=True) * d, axis=1)
    k = int(np.argmin(dist))
    x, y = int(xs.ravel()[k]), int(ys.ravel()[k])
    return (x - 16) & ~1, (y - 16) & ~1


def crop_cfg(name: str, pdf, cdf, sky_configs, sky_radiances):
    """(render configuration dict of the frame, crop origin (x0, y0))."""
    eye, w, h = _frame(name)
    viewi, proji = cam.camera_matrices(eye, W.CENTER, W.CAMERA["fov"], w, h)
    ss, sa, ev = W.medium(CONFIGS[name]["medium"])
    cfg = dict(sigma_s=ss, sigma_a=sa, scattevs=ev, sun_dir=cam.sun_direction(W.SUN["elevation"], W.SUN["azimuth"]),
               sun_color=np.asarray(W.SUN["color"], np.float32), sun_angle=W.SUN["angle"],
               turbidity=W.SKY["turbidity"], ground_albedo=W.SKY["albedo"], sky_configs=sky_configs,
               sky_radiances=sky_radiances, mie_pdf=pdf, mie_cdf=cdf, viewi=viewi, proji=proji, w=w, h=h)
    return cfg, crop_origin(name, viewi, proji, w, h)


def block_stats(img):
    """img (2 buffers, 32, 32, 4) -> (sums per buffer and channel (2, 4), sums
    over the 4x4 blocks of 8x8 pixels (2, 4, 4, 4))."""
    img = np.asarray(img, np.float64)
    return img.sum((1, 2)), img.reshape(2, 4, 8, 4, 8, 4).sum((2, 4))


def max_welch_z(R, Q) -> float:
    """Largest per-statistic Welch |z| of two stacks of independent per-run
    statistics (runs along axis 0)."""
    r, q = np.asarray(R, np.float64), np.asarray(Q, np.float64)
    se = np.sqrt(r.var(0, ddof=1) / len(r) + q.var(0, ddof=1) / len(q))
    diff = np.abs(r.mean(0) - q.mean(0))
    zz = np.where(se > 0, diff / np.where(se > 0, se, 1.0), np.where(diff > 0, np.inf, 0.0))
    return float(zz.max())
