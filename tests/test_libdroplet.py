"""The libdroplet boundary driven by a duck-typed stand-in for Blender's bpy
objects (Blender is not available here), the way addon/__init__.py calls it:
BeginRender -> poll QueryStatus -> Render per tile -> poll QueryResult ->
EndRender (src/main.cpp:64-771)."""
import importlib
import time
from types import SimpleNamespace as NS

import numpy as np
import pytest

from conftest import c0_cfg, golden, mie_table, sky_state_c0
from droplet_b200 import camera as cam
from droplet_b200 import workloads as W


def quat_from_forward(d):
    """Unit quaternion (x, y, z, w) rotating (0, 0, -1) onto direction d."""
    a = np.array([0.0, 0.0, -1.0])
    b = np.asarray(d, np.float64) / np.linalg.norm(d)
    c = np.cross(a, b)
    w = 1.0 + float(np.dot(a, b))
    q = np.array([c[0], c[1], c[2], w])
    return q / np.linalg.norm(q)


class Quat(NS):
    pass


def rot(q):
    return NS(to_quaternion=lambda: Quat(x=q[0], y=q[1], z=q[2], w=q[3]))


def fake_scene(w=64, h=64):
    eye = cam.orbit_eye(W.CENTER, W.CAMERA["distance"], W.CAMERA["azimuth"], W.CAMERA["elevation"])
    near, far = 0.1, 100.0
    t = np.tan(np.radians(W.CAMERA["fov"]) / 2)
    frame = [NS(x=2 * near * t * w / h, y=2 * near * t, z=-near)]
    camera = NS(location=NS(x=eye[0], y=eye[1], z=eye[2]),
                rotation_euler=rot(quat_from_forward(np.asarray(W.CENTER) - eye)),
                data=NS(view_frame=lambda scene: iter(frame), clip_start=near, clip_end=far))
    sd = cam.sun_direction(W.SUN["elevation"], W.SUN["azimuth"]).astype(np.float64)
    lamp = NS(type="LAMP", hide_render=0, rotation_euler=rot(quat_from_forward(-sd)),
              data=NS(droplet=NS(color=NS(r=1.0, g=1.0, b=1.0), intensity=1.0, angle=W.SUN["angle"])))
    ss, sa, ev = W.medium("c0")
    z = golden("c0_octree.npz")
    return NS(camera=camera, objects=[lamp, NS(type="MESH", hide_render=1)],
              blcloudsampling=NS(scatterevs=ev, msigmas=ss, msigmaa=sa, phasef="M", phasea=0.0),
              blcloudgrid=NS(detailsize=1 / 64, qfbandw=0.1, maxdepth=12),
              world=NS(droplet=NS(depthcomp=False, occlusion=False, envtex="(droplet.nan)", depthtex="(droplet.nan)",
                                  turbidity=W.SKY["turbidity"], ground_albedo=W.SKY["albedo"])),
              droplet_volume={"block_origin": z["block_origin"], "block_values": z["block_values"],
                              "voxel_size": 1 / 64})


@pytest.fixture
def lib():
    import libdroplet

    libdroplet = importlib.reload(libdroplet)
    pdf, cdf = mie_table()
    libdroplet.SetPhaseTable(pdf, cdf)
    libdroplet.SetSkyState(*sky_state_c0())
    yield libdroplet
    libdroplet.EndRender()


def wait_ready(lib, timeout=60):
    t = time.time()
    while lib.QueryStatus() != 0:
        assert time.time() - t < timeout
        time.sleep(0.01)


def test_begin_render_parses_the_scene(lib):
    scene = fake_scene()
    lib.BeginRender(scene, NS(), 32, 32, 64, 64, 1)
    job = lib._job
    cfg = c0_cfg(64, 64)
    # the camera built from a Blender camera (LookToRH of the rotated -z axis,
    # PerspectiveRH of the view frame) equals the configuration's matrices
    assert np.allclose(job["viewi"], cfg["viewi"], atol=2e-6)
    assert np.allclose(job["proji"], cfg["proji"], atol=2e-6)
    assert np.allclose(job["sun"][0], cfg["sun_dir"], atol=1e-6)
    assert job["scattevs"] == cfg["scattevs"]
    wait_ready(lib)


def test_begin_render_twice_is_an_error(lib):
    lib.BeginRender(fake_scene(), NS(), 32, 32, 64, 64, 1)
    with pytest.raises(SystemError):
        lib.BeginRender(fake_scene(), NS(), 32, 32, 64, 64, 1)
    wait_ready(lib)


def test_bad_arguments_are_errors(lib):
    with pytest.raises(SystemError):
        lib.BeginRender(fake_scene(), NS(), -1, 32, 64, 64, 1)
    scene = fake_scene()
    scene.objects = []
    with pytest.raises(SystemError, match="lamp"):
        lib.BeginRender(scene, NS(), 32, 32, 64, 64, 1)


def test_no_kernel_without_gpu(lib):
    from droplet_b200 import _native as N

    if N.device_count() > 0:
        pytest.skip("a GPU is present")
    lib.BeginRender(fake_scene(), NS(), 32, 32, 64, 64, 1)
    wait_ready(lib)
    assert "device" in (lib.LastError() or "").lower() or "cuda" in (lib.LastError() or "").lower()
    with pytest.raises(SystemError, match="no render kernel"):
        lib.Render(0, 0, 32, 32, 4)


@pytest.mark.gpu
def test_addon_flow_renders_tiles(lib):
    """Tiles through the module equal the renderer's own tiles (same streams)."""
    from conftest import settings_from_cfg
    from droplet_b200.renderer import Renderer
    from droplet_b200.scene import Octree

    lib.BeginRender(fake_scene(), NS(), 32, 32, 64, 64, 1)
    wait_ready(lib)
    assert lib.LastError() is None
    acc = np.zeros((32 * 32, 4))
    for chunk in range(2):
        lib.Render(16, 16, 32, 32, 8)
        while True:
            qr = lib.QueryResult(0)
            if qr is not None:
                break
        assert len(qr) == 32 * 32 and len(qr[0]) == 4
        acc += qr
        acc += lib.QueryResult(1)
    from conftest import golden_octree

    nodes, bricks, mlevel = golden_octree()
    with Renderer(0) as r:
        r.upload(Octree(nodes, bricks, mlevel))
        r.set_params(settings_from_cfg(c0_cfg(64, 64)))
        ref = np.zeros((32, 32, 4))
        for chunk in range(2):
            a, b = r.render_tile(16, 16, 32, 32, 8)
            ref += a + b
    assert np.allclose(acc, ref.reshape(-1, 4), rtol=1e-3, atol=1e-5 * np.abs(ref).max())


@pytest.mark.gpu
def test_addon_shadow_pass(lib):
    """libdroplet.Shadow as RenderShadow (addon/__init__.py:126-152) drives it:
    QueryResult(0) holds the shadow sums of the tile, equal to the renderer's."""
    from conftest import depth_texture, golden_octree, settings_from_cfg
    from droplet_b200.renderer import Renderer
    from droplet_b200.scene import Octree

    scene = fake_scene()
    scene.droplet_depth = depth_texture(64, 64)
    lib.BeginRender(scene, NS(), 32, 32, 64, 64, 1)
    wait_ready(lib)
    lib.Shadow(8, 8, 32, 32, 100)
    while True:
        qr = lib.QueryResult(0)
        if qr is not None:
            break
    got = np.asarray(qr, np.float64)
    assert got.shape == (32 * 32, 4)
    nodes, bricks, mlevel = golden_octree()
    cfg = c0_cfg(64, 64)
    cfg["depth"] = depth_texture(64, 64)
    with Renderer(0) as r:
        r.upload(Octree(nodes, bricks, mlevel))
        r.set_params(settings_from_cfg(cfg))
        ref, _ = r.render_shadow_tile(8, 8, 32, 32, 100)
    assert np.array_equal(got[:, :3], ref.reshape(-1, 4)[:, :3])
    assert (got[:, :3] < 100).any() and np.isposinf(got[:, 3]).all()


def test_begin_render_reads_occluders_with_the_occlusion_option(lib):
    from conftest import occluder_surfaces

    scene = fake_scene()
    scene.droplet_surfaces = [{"vertices": v, "indices": ix, "holdout": bool(f & 2)} for v, ix, f in occluder_surfaces()]
    lib.BeginRender(scene, NS(), 32, 32, 64, 64, 1)
    assert lib._job["occlusion"] is False and lib._job["surfaces"] == []
    wait_ready(lib)
    lib.EndRender()
    scene.world.droplet.occlusion = True
    lib.BeginRender(scene, NS(), 32, 32, 64, 64, 1)
    job = lib._job
    assert job["occlusion"] is True
    assert [len(ix) for _, ix, _ in job["surfaces"]] == [len(ix) for _, ix, _ in occluder_surfaces()]
    assert [f for _, _, f in job["surfaces"]] == [f for _, _, f in occluder_surfaces()]
    wait_ready(lib)


@pytest.mark.gpu
def test_addon_flow_with_occluders_matches_renderer(lib):
    """With world.droplet.occlusion the module renders what the renderer renders
    with the same occluders and the USE_EMBREE build's masks."""
    from conftest import golden_octree, occluder_surfaces, settings_from_cfg
    from droplet_b200.renderer import Renderer
    from droplet_b200.scene import Octree

    scene = fake_scene()
    scene.world.droplet.occlusion = True
    scene.droplet_surfaces = [{"vertices": v, "indices": ix, "holdout": bool(f & 2)} for v, ix, f in occluder_surfaces()]
    lib.BeginRender(scene, NS(), 32, 32, 64, 64, 1)
    wait_ready(lib)
    lib.Render(16, 16, 32, 32, 16)
    wait_ready(lib)
    assert lib.LastError() is None
    sun = np.asarray(lib.QueryResult(0), np.float64).reshape(32, 32, 4)
    nodes, bricks, mlevel = golden_octree()
    cfg = c0_cfg(64, 64)
    cfg["embree"] = True
    with Renderer(0) as r:
        r.set_occluders(occluder_surfaces())
        r.upload(Octree(nodes, bricks, mlevel))
        r.set_params(settings_from_cfg(cfg))
        ref, _ = r.render_tile(16, 16, 32, 32, 16)
        r.set_occluders([])
        plain, _ = r.render_tile(16, 16, 32, 32, 16, sample_base=0)
    assert np.allclose(sun, ref, rtol=1e-3, atol=1e-5 * np.abs(ref).max())
    assert sun[..., :3].sum() < 0.97 * plain[..., :3].sum()


def test_begin_render_reads_phase_and_environment(lib):
    from test_phase_env import env_map

    scene = fake_scene()
    scene.blcloudsampling.phasef = "H"
    scene.blcloudsampling.phasea = 0.6
    em = env_map()
    scene.world.droplet.envtex = "sky.exr"
    data = NS(images={"sky.exr": NS(size=(em.shape[1], em.shape[0]), pixels=em.reshape(-1).tolist())})
    lib.BeginRender(scene, data, 32, 32, 64, 64, 1)
    job = lib._job
    assert job["phase"] == ("hg", 0.6)
    assert job["env"] is None  # the Hosek build reads no environment texture
    wait_ready(lib)
    lib.EndRender()
    lib.SetSkyModel("environment")
    lib.BeginRender(scene, data, 32, 32, 64, 64, 1)
    assert np.array_equal(lib._job["env"], em)
    wait_ready(lib)
    with pytest.raises(SystemError):
        lib.SetSkyModel("other")
