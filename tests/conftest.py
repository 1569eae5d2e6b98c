"""Shared test setup.

Markers: `gpu` tests need a B200 and call the product through its C ABI; the
rest run on the CPU (oracle pins, host builder, library loading, boundary).
The CPU checkers live in oracle/ (test infrastructure only).
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "droplet-render_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

from droplet_b200 import camera as cam  # noqa: E402
from droplet_b200 import workloads as W  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); calls the product through its C ABI")


def golden(name: str):
    path = os.path.join(GOLDEN, name)
    if name.endswith(".json"):
        with open(path) as f:
            return json.load(f)
    with np.load(path) as z:  # materialise: NpzFile re-reads members on each access
        return {k: np.ascontiguousarray(z[k]) for k in z.files}


def golden_octree():
    from oracle.oracle import NODE_DTYPE

    z = golden("c0_octree.npz")
    return z["nodes"].view(NODE_DTYPE).reshape(-1), z["bricks"], int(z["mlevel"].reshape(-1)[0])


def mie_table():
    z = golden("mie_reference_table.npz")
    return np.ascontiguousarray(z["pdf"], np.float32), np.ascontiguousarray(z["cdf"], np.float32)


def sky_state_c0():
    for s in golden("sky_states.json"):
        if s["note"] == "c0/c1 sun":
            return np.asarray(s["configs"], np.float64), np.asarray(s["radiances"], np.float64)
    raise KeyError("c0 sky state")


def c0_cfg(w: int, h: int, medium: str = "c0") -> dict:
    """Render configuration dict for config 0 at w x h (inputs from the fixtures)."""
    pdf, cdf = mie_table()
    cfgs, rads = sky_state_c0()
    sd = cam.sun_direction(W.SUN["elevation"], W.SUN["azimuth"])
    eye = cam.orbit_eye(W.CENTER, W.CAMERA["distance"], W.CAMERA["azimuth"], W.CAMERA["elevation"])
    viewi, proji = cam.camera_matrices(eye, W.CENTER, W.CAMERA["fov"], w, h)
    ss, sa, ev = W.medium(medium)
    return dict(sigma_s=ss, sigma_a=sa, scattevs=ev, sun_dir=sd, sun_color=np.asarray(W.SUN["color"], np.float32),
                sun_angle=W.SUN["angle"], turbidity=W.SKY["turbidity"], ground_albedo=W.SKY["albedo"],
                sky_configs=cfgs, sky_radiances=rads, mie_pdf=pdf, mie_cdf=cdf, viewi=viewi, proji=proji, w=w, h=h)


def settings_from_cfg(cfg: dict):
    from droplet_b200.renderer import PhaseTable, RenderSettings
    from droplet_b200.sky import SkyState

    return RenderSettings(
        sigma_s=cfg["sigma_s"], sigma_a=cfg["sigma_a"], scattevs=cfg["scattevs"], sun_dir=cfg["sun_dir"],
        sun_color=cfg["sun_color"], sun_angle=cfg["sun_angle"],
        sky=SkyState(np.asarray(cfg["sky_configs"]), np.asarray(cfg["sky_radiances"])),
        phase=PhaseTable(cfg["mie_pdf"], cfg["mie_cdf"]), viewi=cfg["viewi"], proji=cfg["proji"], w=cfg["w"],
        h=cfg["h"], depth=cfg.get("depth"), depthcomp=bool(cfg.get("depthcomp", False)),
        finite_paths=bool(cfg.get("finite_paths", False)),
        embree=bool(cfg.get("embree", False)),
        phase_mode=int(cfg.get("phase_mode", 0)), hg_g=float(cfg.get("hg_g", 0.0)),
        env_mode=int(cfg.get("env_mode", 0)), env_map=cfg.get("env_map"))


def depth_texture(w: int, h: int) -> np.ndarray:
    """Depth texture for the shadow-pass and compositing checks: every third pixel
    has no geometry before the far plane (1e30), the others sit 2.3-2.7 units
    along the camera ray (inside the config-0 cloud, 2.5 units from the camera)."""
    j, i = np.mgrid[0:h, 0:w]
    d = (2.3 + 0.4 * ((i * 7 + j * 3) % 11) / 10.0).astype(np.float32)
    d[(i + j) % 3 == 0] = np.float32(1e30)
    return d


def clip_end(proji) -> np.float32:
    """Far clip distance of RenderKernel::Shadow: -z/w of (0,0,1,1) * projInv."""
    q = np.asarray(proji, np.float32).reshape(4, 4)
    return np.float32(-np.float32(q[2, 2] + q[3, 2]) / np.float32(q[2, 3] + q[3, 3]))


@pytest.fixture(scope="session")
def port():
    from oracle import Port, port_available

    if not port_available():
        pytest.skip("oracle port not built (make -C oracle port)")
    return Port()


@pytest.fixture(scope="session")
def ref():
    from oracle import Reference, ref_available

    if not ref_available():
        pytest.skip("reference oracle not built (needs the reference sources; make -C oracle ref)")
    return Reference()


@pytest.fixture(scope="session")
def c0_octree():
    return golden_octree()


@pytest.fixture(scope="session")
def gpu_renderer():
    """A renderer on cuda:0 with the config-0 scene and 64x64 parameters."""
    from droplet_b200.renderer import Renderer
    from droplet_b200.scene import Octree

    nodes, bricks, mlevel = golden_octree()
    r = Renderer(0)
    r.upload(Octree(nodes.view(np.uint8).view(nodes.dtype), bricks, mlevel))
    r.set_params(settings_from_cfg(c0_cfg(64, 64)))
    yield r
    r.close()


# A path of the reference estimator whose sky term is 0/0: in the uniform
# 0.3 cube (128^3), camera at azimuth 0 (256 x 256), pixel (131, 158),
# stream (1000 + 0x9E3779B9, pixel, 9) escapes at r = 4 along a direction
# with rd.y == 0 exactly.
NAN_PATH = {"pixel": (131, 158), "seed": 1000 + 0x9E3779B9, "sample": 9}


def uniform_cube_scene(build):
    """The uniform 0.3 grid of 128^3 as (nodes, bricks, mlevel) from `build`
    (a builder taking block origins, values, voxel size, maxdepth)."""
    from droplet_b200 import workloads as W

    org, vals = W.dense_to_blocks(np.full((128, 128, 128), 0.3, np.float32))
    return build(org, vals, 1 / 128, 12)


def orbit_cfg(w: int, h: int, azimuth: float) -> dict:
    cfg = c0_cfg(w, h)
    eye = cam.orbit_eye(W.CENTER, W.CAMERA["distance"], azimuth, W.CAMERA["elevation"])
    cfg["viewi"], cfg["proji"] = cam.camera_matrices(eye, W.CENTER, W.CAMERA["fov"], w, h)
    return cfg


def occluder_surfaces():
    """Occluder meshes around the config-0 cloud, as (vertices, indices, flags):
    a holdout UV sphere (radius 0.25) between the cloud and the sun, a ground
    quad (z = 0.02, not flagged holdout) under it, and 200 small holdout
    triangles beside it (seeded)."""
    sd = cam.sun_direction(W.SUN["elevation"], W.SUN["azimuth"]).astype(np.float64)
    c = np.asarray(W.CENTER) + 0.9 * sd
    nu, nv = 24, 12
    th = np.linspace(0.0, np.pi, nv + 1)
    ph = np.linspace(0.0, 2 * np.pi, nu, endpoint=False)
    verts = [c + 0.25 * np.array([np.sin(t) * np.cos(p), np.sin(t) * np.sin(p), np.cos(t)]) for t in th for p in ph]
    tris = []
    for i in range(nv):
        for j in range(nu):
            a, b = i * nu + j, i * nu + (j + 1) % nu
            d, e = (i + 1) * nu + j, (i + 1) * nu + (j + 1) % nu
            tris += [(a, d, b), (b, d, e)]
    sphere = (np.asarray(verts, np.float32), np.asarray(tris, np.uint32), 0x2)
    ground = (np.array([[-20, -20, 0.02], [20, -20, 0.02], [20, 20, 0.02], [-20, 20, 0.02]], np.float32),
              np.array([[0, 1, 2], [0, 2, 3]], np.uint32), 0x0)
    rng = np.random.default_rng(31)
    base = rng.uniform([1.1, 0.0, 0.0], [1.6, 1.0, 1.0], (200, 3))
    v = (base[:, None, :] + rng.normal(scale=0.05, size=(200, 3, 3))).reshape(-1, 3).astype(np.float32)
    small = (v, np.arange(600, dtype=np.uint32).reshape(-1, 3), 0x2)
    return [sphere, ground, small]


def sdf_scene(radius: float = 0.18):
    """The config-0 octree with an opaque sphere (centre (0.5, 0.5, 0.5)):
    leaves within 1.5 leaf diagonals of its surface get an SDF brick (signed
    distance at the brick's sample positions, the resampling of
    src/scene.cpp:880-886), every third of those loses its fog brick, and
    fog leaves wholly inside the sphere are removed as the reference's builder
    removes them (src/scene.cpp:875-883).  Returns (nodes, bricks, sdf_bricks,
    mlevel)."""
    from oracle.oracle import NODE_DTYPE

    nodes, bricks, mlevel = golden_octree()
    nodes = nodes.copy()
    c = np.array(W.CENTER, np.float64)
    vol = nodes["volx"]
    leaves = np.flatnonzero((vol[:, 0] != 0xFFFFFFFF) | (vol[:, 1] != 0xFFFFFFFF))
    sdf = []
    t = (8.0 - 2.0 * np.arange(8) - 1.0) / 7.0
    for k, i in enumerate(leaves):
        ce = nodes["ce"][i].astype(np.float64)
        d = np.linalg.norm(ce[:3] - c) - radius
        diag = np.sqrt(3.0) * ce[3]
        if d < -1.5 * diag:
            nodes["volx"][i, 1] = 0xFFFFFFFF  # inside the surface: no fog leaf
            continue
        if abs(d) > 1.5 * diag:
            continue
        z, y, x = np.meshgrid(t, t, t, indexing="ij")  # brick order: x fastest
        p = np.stack([ce[0] - ce[3] * x, ce[1] - ce[3] * y, ce[2] - ce[3] * z], -1).reshape(-1, 3)
        sdf.append((np.linalg.norm(p - c, axis=1) - radius).astype(np.float32))
        nodes["volx"][i, 0] = len(sdf) - 1
        if len(sdf) % 3 == 0:
            nodes["volx"][i, 1] = 0xFFFFFFFF  # surface leaf without fog
    assert nodes.dtype == NODE_DTYPE
    return nodes, bricks, np.ascontiguousarray(np.stack(sdf)), mlevel
