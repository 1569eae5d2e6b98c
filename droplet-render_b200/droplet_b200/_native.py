"""ctypes binding of the droplet_b200 C ABI (include/droplet_b200.h).

The shared library is built in-tree (droplet_b200/_lib/libdroplet_b200.so,
see csrc/Makefile).  Loading fails loudly when it is missing: there is no
CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libdroplet_b200.so")

DR_OK = 0
DR_ERR_INVALID = -1
DR_ERR_CUDA = -2
DR_ERR_STATE = -3
DR_ERR_NOMEM = -4
DR_ERR_GAVE_UP = -5
DR_ERR_NODEVICE = -6
DR_NONE = 0xFFFFFFFF

DR_PHASE_MIE_REFERENCE = 0
DR_PHASE_MIE_EXACT = 1
DR_PHASE_HG = 2
DR_ENV_HOSEK = 0
DR_ENV_NONE = 1
DR_ENV_MAP = 2
DR_VERSION = 200  # include/droplet_b200.h: the struct layouts below
DR_KERNEL_DEPTHCOMP = 0x1
DR_KERNEL_FINITE_PATHS = 0x2
DR_KERNEL_EMBREE = 0x4

DR_PROBE_MIE_EVAL_RGB = 0
DR_PROBE_MIE_SAMPLE = 1
DR_PROBE_SUN_SAMPLE = 2
DR_PROBE_SKY = 3
DR_PROBE_MIE_THETA = 4
DR_PROBE_MIE_EXACT_DIR = 5
DR_PROBE_HG_EVAL = 6
DR_PROBE_HG_SAMPLE = 7
DR_PROBE_SKY_LIGHT = 8
DR_PROBE_ENV_MAP = 9


class DrError(RuntimeError):
    """A droplet_b200 call returned an error code."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"droplet_b200 error {code}: {msg}")
        self.code = code


class DrGaveUp(DrError):
    """DR_ERR_GAVE_UP: the call finished, but some paths were cut short by an
    iteration budget, so its outputs are incomplete.  `result` holds the
    outputs where the raising method has them (else None)."""

    result = None


class DrNode(C.Structure):
    """Octree node record, the reference's OctreeStructure (src/scene.h:21-31)."""

    _fields_ = [("ce", C.c_float * 4), ("chn", C.c_uint32 * 8), ("volx", C.c_uint32 * 2), ("qval", C.c_float * 2)]


class DrOctree(C.Structure):
    _fields_ = [
        ("nodes", C.POINTER(DrNode)),
        ("n_nodes", C.c_uint32),
        ("bricks", C.POINTER(C.c_float)),
        ("n_leaves", C.c_uint32),
        ("lvoxc", C.c_uint32),
        ("mlevel", C.c_uint32),
    ]


class DrSceneDesc(C.Structure):
    _fields_ = [
        ("nodes", C.c_void_p),
        ("n_nodes", C.c_uint32),
        ("bricks", C.c_void_p),
        ("n_leaves", C.c_uint32),
        ("lvoxc", C.c_uint32),
        ("sdf_bricks", C.c_void_p),
        ("n_sdf_leaves", C.c_uint32),
    ]


class DrSurface(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("n_vertices", C.c_uint32), ("indices", C.c_void_p),
                ("n_triangles", C.c_uint32), ("flags", C.c_uint32)]


class DrRenderParams(C.Structure):
    _fields_ = [
        ("sigma_s", C.c_float),
        ("sigma_a", C.c_float),
        ("scattevs", C.c_uint32),
        ("sun_dir", C.c_float * 3),
        ("sun_color", C.c_float * 3),
        ("sun_angle", C.c_float),
        ("sky_configs", (C.c_double * 9) * 3),
        ("sky_radiances", C.c_double * 3),
        ("mie_pdf", C.c_void_p),
        ("mie_cdf", C.c_void_p),
        ("mie_n", C.c_uint32),
        ("phase_mode", C.c_uint32),
        ("viewi", C.c_float * 16),
        ("proji", C.c_float * 16),
        ("w", C.c_uint32),
        ("h", C.c_uint32),
        ("depth", C.c_void_p),
        ("flags", C.c_uint32),
        ("hg_g", C.c_float),
        ("env_mode", C.c_uint32),
        ("env_map", C.c_void_p),
        ("env_w", C.c_uint32),
        ("env_h", C.c_uint32),
    ]


class DrCounters(C.Structure):
    _fields_ = [
        ("paths", C.c_uint64),
        ("vertices", C.c_uint64),
        ("node_visits", C.c_uint64),
        ("density_lookups", C.c_uint64),
        ("mie_evals", C.c_uint64),
        ("gave_up", C.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {f: int(getattr(self, f)) for f, _ in self._fields_}


class DrTuning(C.Structure):
    _fields_ = [("kernel", C.c_uint32), ("blocks_per_sm", C.c_uint32), ("event_batch", C.c_uint32),
                ("traversal", C.c_uint32), ("tile", C.c_uint32), ("visits", C.c_uint32), ("steps", C.c_uint32)]


class DrBatchView(C.Structure):
    _fields_ = [("scene", C.c_uint32), ("params", C.c_void_p), ("x0", C.c_uint32), ("y0", C.c_uint32),
                ("tw", C.c_uint32), ("th", C.c_uint32), ("spp", C.c_uint32), ("seed", C.c_uint64)]


# name -> (restype, argtypes); every symbol the header declares
SIGNATURES = {
    "dr_version": (C.c_int, []),
    "dr_last_error": (C.c_char_p, []),
    "dr_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "dr_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "dr_destroy": (C.c_int, [C.c_void_p]),
    "dr_build_octree": (
        C.c_int,
        [C.c_void_p, C.c_void_p, C.c_uint32, C.c_float, C.c_uint32, C.c_int, C.POINTER(DrOctree)],
    ),
    "dr_octree_free": (None, [C.POINTER(DrOctree)]),
    "dr_upload_scene": (C.c_int, [C.c_void_p, C.POINTER(DrSceneDesc)]),
    "dr_set_occluders": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32]),
    "dr_build_occluder_bvh": (
        C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.POINTER(C.c_uint32), C.c_void_p, C.c_void_p,
                  C.POINTER(C.c_uint32)]),
    "dr_set_params": (C.c_int, [C.c_void_p, C.POINTER(DrRenderParams)]),
    "dr_sky_cook": (
        C.c_int,
        [C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_void_p],
    ),
    "dr_render_tile": (
        C.c_int,
        [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64, C.c_void_p,
         C.c_void_p],
    ),
    "dr_render_tile_async": (
        C.c_int,
        [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64, C.c_void_p,
         C.c_void_p, C.c_void_p],
    ),
    "dr_shadow_tile": (
        C.c_int,
        [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64, C.c_void_p],
    ),
    "dr_shadow_tile_async": (
        C.c_int,
        [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64, C.c_void_p,
         C.c_void_p],
    ),
    "dr_synchronize": (C.c_int, [C.c_void_p]),
    "dr_check_complete": (C.c_int, [C.c_void_p, C.c_void_p]),
    "dr_set_step_budget": (C.c_int, [C.c_void_p, C.c_uint32]),
    "dr_set_camera_lists": (C.c_int, [C.c_void_p, C.c_uint32]),
    "dr_set_bricks_dev": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_float, C.c_void_p]),
    "dr_get_majorants": (C.c_int, [C.c_void_p, C.c_void_p]),
    "dr_adjoint_tile_async": (
        C.c_int,
        [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64, C.c_void_p,
         C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    ),
    "dr_reweighted_loss_async": (
        C.c_int,
        [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64, C.c_void_p,
         C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    ),
    "dr_adjoint_transmittance": (
        C.c_int,
        [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p],
    ),
    "dr_batch_create": (
        C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p)]),
    "dr_batch_destroy": (C.c_int, [C.c_void_p]),
    "dr_batch_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(DrTuning)]),
    "dr_batch_get_tuning": (C.c_int, [C.c_void_p, C.POINTER(DrTuning)]),
    "dr_batch_launch": (C.c_int, [C.c_void_p, C.c_void_p]),
    "dr_batch_output": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "dr_batch_read": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    "dr_batch_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "dr_batch_set_split": (C.c_int, [C.c_void_p, C.c_uint64]),
    "dr_batch_get_split": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)]),
    "dr_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(DrTuning)]),
    "dr_get_tuning": (C.c_int, [C.c_void_p, C.POINTER(DrTuning)]),
    "dr_get_counters": (C.c_int, [C.c_void_p, C.POINTER(DrCounters)]),
    "dr_reset_counters": (C.c_int, [C.c_void_p]),
    "dr_probe_leaf_sequence": (
        C.c_int,
        [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    ),
    "dr_probe_density": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "dr_probe_occlusion": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "dr_probe_paths": (
        C.c_int,
        [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p],
    ),
    "dr_probe_sampler": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p]),
    "dr_probe_transmittance": (
        C.c_int,
        [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint64, C.c_void_p],
    ),
    "dr_transmittance_noalloc": (
        C.c_int,
        [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p],
    ),
}

DR_NOALLOC_MAX_RAYS = 65536

_lib = None
_lock = threading.Lock()


def lib() -> C.CDLL:
    """The loaded library; raises if the in-tree build is missing."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"droplet_b200 native library not built: {LIB_PATH} is missing "
                    "(run `make -C droplet-render_b200/csrc` or __graft_entry__.build())"
                )
            L = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            if L.dr_version() != DR_VERSION:
                raise ImportError(f"{LIB_PATH} has interface version {L.dr_version()}, this binding expects "
                                  f"{DR_VERSION}: rebuild the library")
            _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != DR_OK:
        msg = lib().dr_last_error().decode(errors="replace")
        raise (DrGaveUp if rc == DR_ERR_GAVE_UP else DrError)(rc, msg)


def device_count() -> int:
    n = C.c_int(0)
    rc = lib().dr_device_count(C.byref(n))
    if rc == DR_ERR_NODEVICE:
        return 0
    check(rc)
    return int(n.value)
