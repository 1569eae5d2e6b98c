"""libdroplet: the native-module interface the droplet-render Blender addon
imports (addon/__init__.py:17), backed by the droplet_b200 GPU renderer.

Same six functions, argument meanings, asynchronous behaviour and error
behaviour as the reference module (src/main.cpp:64-771):

  BeginRender(scene, data, tilex, tiley, w, h, smask)  src/main.cpp:64-648
      reads the camera, lamps and render properties from the Blender scene and
      builds the volume on a background thread (QueryStatus() == 1 until done)
  Render(x0, y0, tilew, tileh, samples)                 src/main.cpp:650-667
      renders one tile on a background thread; ignored while busy
  Shadow(x0, y0, tilew, tileh, samples)                 src/main.cpp:669-686
  QueryStatus() -> 0 ready / 1 processing               src/main.cpp:718-721
  QueryResult(bindex) -> None while busy, else a list of [r, g, b, a] per
      pixel of the last tile: bindex 0 = sun, 1 = sky; sums over the samples
      of the last call                                   src/main.cpp:723-746
  EndRender()                                            src/main.cpp:688-716

Where the reference returns NULL (invalid arguments, no kernel), Python sees a
SystemError; the same exception type is raised here, with a message.

Inputs the reference takes from places outside the rendering path:
  * the volume: the reference evaluates Blender node trees into OpenVDB grids
    (src/scene.cpp, SceneDensity.cpp), which is not part of this library.  The
    scene object passed to BeginRender must carry `droplet_volume`, either
    {"grid": dense ndarray indexed [x, y, z], "voxel_size": s} or
    {"block_origin": (B, 3) int, "block_values": (B, 512) float, "voxel_size": s};
  * the Mie table (compiled into the reference, src/KernelSampler.cpp:8-141):
    SetPhaseTable(pdf, cdf) or the DROPLET_MIE_TABLE environment variable (an
    .npz with arrays pdf and cdf);
  * the Hosek-Wilkie RGB dataset for the sky cook (compiled into the
    reference): SetSkyDataset(path) or DROPLET_HOSEK_DATASET (the model's C
    header), or SetSkyState(configs, radiances).  Turbidity and ground albedo
    are read from world.droplet.turbidity / ground_albedo when present, else
    the reference's fixed 7 and 0.15 (src/kernel.cpp:525);
  * the phase function: blcloudsampling.phasef 'M' (Mie) or 'H' (Henyey-
    Greenstein with phasea), as src/main.cpp:522-536;
  * the environment: by default escaping rays take the Hosek sky (the
    reference built with USE_ARHOSEK_SKYMODEL); SetSkyModel("environment")
    selects its default build, whose light is the world.droplet.envtex image
    (MapEnv) or none (NullEnv);
  * occlusion geometry: with world.droplet.occlusion set, the reference (built
    with Embree) occludes with the triangle meshes its node trees produce
    (SceneData::Surface, src/main.cpp:406-419, src/SceneOcclusion.cpp:19-56).
    Here they come from `scene.droplet_surfaces`, a list of
    {"vertices": (n, 3), "indices": (m, 3), "holdout": bool}; every surface
    occludes, as in the reference, unless SetOccluderMode(holdout_only=True).
"""
from __future__ import annotations

import os
import sys
import threading
import traceback

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
if _HERE not in sys.path:
    sys.path.insert(0, _HERE)

from droplet_b200 import camera as _cam  # noqa: E402

ENGINE_STATE_READY = 0
ENGINE_STATE_PROCESSING = 1

_lock = threading.RLock()
_state = ENGINE_STATE_READY
_renderer = None          # droplet_b200.renderer.Renderer once the scene is built
_scene_built = False
_build_error = None
_job = None               # dict describing the parsed scene
_tile = None              # (sun, sky) arrays of the last Render/Shadow call
_tile_error = None        # why the last Render/Shadow call produced no complete tile
_tile_size = (0, 0)
_phase = None
_sky_dataset = None
_sky_state = None
_holdout_only = False     # occluders: every surface (the reference) or holdout meshes only
_sky_model = "hosek"      # "hosek": the reference built with USE_ARHOSEK_SKYMODEL; "environment": its default build
_device = int(os.environ.get("DROPLET_DEVICE", "0"))


def _fail(msg: str):
    raise SystemError(f"libdroplet: {msg}")


# ---- extensions: inputs the reference compiles in ---------------------------
def SetPhaseTable(pdf, cdf):
    global _phase
    _phase = (np.ascontiguousarray(pdf, np.float32).reshape(-1, 3), np.ascontiguousarray(cdf, np.float32).reshape(-1, 3))


def SetSkyDataset(path: str):
    global _sky_dataset
    from droplet_b200 import sky

    _sky_dataset = sky.load_dataset(path)


def SetSkyState(configs, radiances):
    global _sky_state
    from droplet_b200.sky import SkyState

    _sky_state = SkyState(np.asarray(configs, np.float64).reshape(3, 9), np.asarray(radiances, np.float64).reshape(3))


def SetSkyModel(model: str):
    """"hosek" (default): escaping rays take the Hosek-Wilkie sky, as the
    reference built with USE_ARHOSEK_SKYMODEL; "environment": its default
    build, where they take pow(world.droplet.envtex, 2.2) (MapEnv) or nothing
    (NullEnv) when no texture is set (src/kernel.cpp:329-364)."""
    global _sky_model
    if model not in ("hosek", "environment"):
        _fail("sky model must be 'hosek' or 'environment'")
    _sky_model = model


def SetOccluderMode(holdout_only: bool):
    """False (default): every surface occludes, as the reference's
    `!flags & SCENEOBJ_HOLDOUT` test makes it (src/SceneOcclusion.cpp:27);
    True: only surfaces marked holdout, the option's documented intent."""
    global _holdout_only
    _holdout_only = bool(holdout_only)


def LastError():
    return _build_error


# ---- helpers ------------------------------------------------------------------
def _rotate(v, q):
    """Rotates vector v by the unit quaternion q = (x, y, z, w) (XMVector3Rotate)."""
    x, y, z, w = q
    u = np.array([x, y, z], np.float64)
    v = np.asarray(v, np.float64)
    return v + 2.0 * np.cross(u, np.cross(u, v) + w * v)


def _quat(obj):
    q = obj.rotation_euler.to_quaternion()
    return (float(q.x), float(q.y), float(q.z), float(q.w))


def _parse(scene, data, tilex, tiley, w, h):
    cam = scene.camera
    loc = cam.location
    p = np.array([float(loc.x), float(loc.y), float(loc.z)])
    u = np.array([0.0, 0.0, -1.0])
    d = _rotate(u, _quat(cam))
    frame = next(iter(cam.data.view_frame(scene)))
    frx, fry = float(frame.x), float(frame.y)
    zmin, zmax = float(cam.data.clip_start), float(cam.data.clip_end)
    view = _cam.look_to_rh(p, d, u)
    proj = _cam.perspective_rh(frx, fry, zmin, zmax)
    viewi = np.linalg.inv(view).astype(np.float32).reshape(16)
    proji = np.linalg.inv(proj).astype(np.float32).reshape(16)

    suns = []
    for obj in scene.objects:
        if int(getattr(obj, "hide_render", 0)) != 0:
            continue
        if str(obj.type).upper() == "LAMP":
            dd = _rotate(u, _quat(obj))
            sd = obj.data.droplet
            col = np.array([float(sd.color.r), float(sd.color.g), float(sd.color.b)], np.float32)
            suns.append(((-dd).astype(np.float32), (np.float32(float(sd.intensity)) * col).astype(np.float32),
                         float(sd.angle)))
    if not suns:
        _fail("the scene needs a lamp (the reference samples lights[0], src/kernel.cpp:394)")

    sam = scene.blcloudsampling
    phasef = str(sam.phasef)
    # src/main.cpp:522-536: 'H' = HGPhase with g1 = phasea, 'M' = MiePhase
    if phasef[:1] == "H":
        phase = ("hg", float(sam.phasea))
    elif phasef[:1] == "M":
        phase = ("mie", 0.0)
    else:
        _fail(f"unknown phase function {phasef!r}")
    grid = scene.blcloudgrid
    world = scene.world.droplet
    vol = getattr(scene, "droplet_volume", None)
    if vol is None:
        _fail("scene.droplet_volume is missing (the node-tree/OpenVDB volume build is outside this library)")
    # depth texture (src/main.cpp:596-614): read whenever one is supplied; camera
    # rays stop at it only with depthcomp (KERNEL_DEPTHCOMP, src/main.cpp:635)
    depth = None
    if getattr(scene, "droplet_depth", None) is not None:
        depth = np.ascontiguousarray(scene.droplet_depth, np.float32).reshape(h, w)
    depthcomp = bool(getattr(world, "depthcomp", False))
    occlusion = bool(getattr(world, "occlusion", False))
    # environment texture (src/main.cpp:552-587): read by the reference's default
    # build only (without USE_ARHOSEK_SKYMODEL); see SetSkyModel
    env = None
    envtex = str(getattr(world, "envtex", "(droplet.nan)"))
    if _sky_model == "environment" and envtex != "(droplet.nan)":
        img = data.images[envtex] if data is not None and hasattr(data, "images") else None
        if img is not None:
            ew, eh = int(img.size[0]), int(img.size[1])
            env = np.asarray(list(img.pixels), np.float32).reshape(eh, ew, 4)
    surfaces = []
    if occlusion:
        for srf in getattr(scene, "droplet_surfaces", None) or []:
            surfaces.append((np.ascontiguousarray(srf["vertices"], np.float32).reshape(-1, 3),
                             np.ascontiguousarray(srf["indices"], np.uint32).reshape(-1, 3),
                             0x2 if srf.get("holdout") else 0x0))
    return {
        "phase": phase, "env": env,
        "occlusion": occlusion, "surfaces": surfaces,
        "viewi": viewi, "proji": proji, "w": int(w), "h": int(h), "tilex": int(tilex), "tiley": int(tiley),
        "sun": suns[0], "scattevs": int(sam.scatterevs), "sigma_s": float(sam.msigmas), "sigma_a": float(sam.msigmaa),
        "maxdepth": int(grid.maxdepth), "volume": vol, "depth": depth, "depthcomp": depthcomp,
        "turbidity": float(getattr(world, "turbidity", 7.0)), "ground_albedo": float(getattr(world, "ground_albedo", 0.15)),
    }


def _phase_table():
    if _phase is not None:
        return _phase
    path = os.environ.get("DROPLET_MIE_TABLE")
    if not path:
        _fail("no Mie table: call SetPhaseTable(pdf, cdf) or set DROPLET_MIE_TABLE")
    z = np.load(path)
    return np.ascontiguousarray(z["pdf"], np.float32), np.ascontiguousarray(z["cdf"], np.float32)


def _sky(sun_dir, turbidity, albedo):
    from droplet_b200 import sky

    if _sky_state is not None:
        return _sky_state
    ds = _sky_dataset
    if ds is None:
        path = os.environ.get("DROPLET_HOSEK_DATASET")
        if not path:
            _fail("no sky: call SetSkyState/SetSkyDataset or set DROPLET_HOSEK_DATASET")
        ds = sky.load_dataset(path)
    return sky.cook(ds, turbidity, albedo, sky.solar_elevation(sun_dir))


def _build(job):
    """Background part of BeginRender: volume build, GPU context, upload, parameters."""
    global _renderer, _scene_built, _build_error, _state
    try:
        from droplet_b200.renderer import PhaseTable, Renderer, RenderSettings
        from droplet_b200.scene import build_from_dense, build_octree

        vol = job["volume"]
        if "grid" in vol:
            oc = build_from_dense(np.asarray(vol["grid"], np.float32), float(vol["voxel_size"]), job["maxdepth"])
        else:
            oc = build_octree(vol["block_origin"], vol["block_values"], float(vol["voxel_size"]), job["maxdepth"])
        pdf, cdf = _phase_table()
        sd, sc, sa = job["sun"]
        from droplet_b200 import _native as N

        kind, g = job["phase"]
        hosek = _sky_model == "hosek"
        if hosek:
            sky_state = _sky(sd, job["turbidity"], job["ground_albedo"])
        else:
            from droplet_b200.sky import SkyState

            sky_state = SkyState(np.zeros((3, 9)), np.zeros(3))  # unused without the Hosek model
        env_mode = N.DR_ENV_HOSEK if hosek else (N.DR_ENV_MAP if job["env"] is not None else N.DR_ENV_NONE)
        st = RenderSettings(sigma_s=job["sigma_s"], sigma_a=job["sigma_a"], scattevs=job["scattevs"], sun_dir=sd,
                            sun_color=sc, sun_angle=sa, sky=sky_state, phase=PhaseTable(pdf, cdf),
                            viewi=job["viewi"], proji=job["proji"], w=job["w"], h=job["h"], depth=job["depth"],
                            depthcomp=job["depthcomp"], embree=job["occlusion"],
                            phase_mode=N.DR_PHASE_HG if kind == "hg" else N.DR_PHASE_MIE_REFERENCE, hg_g=g,
                            env_mode=env_mode, env_map=job["env"])
        r = Renderer(_device)
        if job["occlusion"]:
            r.set_occluders(job["surfaces"], 1 if _holdout_only else 0)
        r.upload(oc)
        r.set_params(st)
        with _lock:
            _renderer = r
            _scene_built = True
    except Exception as e:  # reported through LastError(); Render then raises SystemError
        with _lock:
            _build_error = f"{type(e).__name__}: {e}"
            if os.environ.get("DROPLET_VERBOSE"):
                traceback.print_exc()
    finally:
        with _lock:
            _state = ENGINE_STATE_READY


def BeginRender(scene, data, tilex, tiley, w, h, smask):
    global _state, _job, _build_error, _scene_built
    with _lock:
        if _job is not None:
            _fail("invalid arguments: a scene is already loaded (call EndRender first)")
        for v in (tilex, tiley, w, h, smask):
            if not isinstance(v, (int, np.integer)) or v < 0:
                _fail("invalid arguments")
        _job = _parse(scene, data, tilex, tiley, w, h)
        _build_error = None
        _scene_built = False
        _state = ENGINE_STATE_PROCESSING
    threading.Thread(target=_build, args=(_job,), daemon=True).start()
    return None


def _tile_worker(kind, x0, y0, tw, th, samples):
    global _tile, _tile_size, _state, _build_error, _tile_error
    try:
        if kind == "render":
            sun, sky = _renderer.render_tile(x0, y0, tw, th, samples)
        else:
            sun, sky = _renderer.render_shadow_tile(x0, y0, tw, th, samples)
        with _lock:
            _tile = (sun.reshape(-1, 4), sky.reshape(-1, 4))
            _tile_size = (tw, th)
    except Exception as e:  # QueryResult raises it (a partial tile is not returned as if complete)
        with _lock:
            _build_error = f"{type(e).__name__}: {e}"
            _tile_error = _build_error
            _tile = None
    finally:
        with _lock:
            _state = ENGINE_STATE_READY


def _start_tile(kind, x0, y0, tilew, tileh, samples):
    global _state, _tile_error
    for v in (x0, y0, tilew, tileh, samples):
        if not isinstance(v, (int, np.integer)) or v < 0:
            _fail("invalid arguments")
    with _lock:
        if _renderer is None:
            if _state == ENGINE_STATE_READY:
                _fail("no render kernel" + (f" ({_build_error})" if _build_error else ""))
            return None  # still building: the reference returns without rendering
        if _state != ENGINE_STATE_READY:
            return None
        _state = ENGINE_STATE_PROCESSING
        _tile_error = None
    threading.Thread(target=_tile_worker, args=(kind, x0, y0, tilew, tileh, samples), daemon=True).start()
    return None


def Render(x0, y0, tilew, tileh, samples):
    return _start_tile("render", x0, y0, tilew, tileh, samples)


def Shadow(x0, y0, tilew, tileh, samples):
    return _start_tile("shadow", x0, y0, tilew, tileh, samples)


def QueryStatus():
    return _state


def QueryResult(bindex):
    with _lock:
        if _renderer is None and _state == ENGINE_STATE_READY:
            _fail("no render kernel")
        if _state != ENGINE_STATE_READY:
            return None
        if not isinstance(bindex, (int, np.integer)) or bindex not in (0, 1):
            _fail("invalid arguments")
        if _tile_error is not None:
            _fail(f"the last Render/Shadow call failed: {_tile_error}")
        if _tile is None:
            return []
        return _tile[bindex].tolist()


def EndRender():
    global _renderer, _job, _tile, _scene_built, _state, _build_error, _tile_error
    with _lock:
        if _renderer is not None:
            _renderer.close()
        _renderer = None
        _job = None
        _tile = None
        _scene_built = False
        _build_error = None
        _tile_error = None
        _state = ENGINE_STATE_READY
    return None
