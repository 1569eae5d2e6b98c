"""The plain single-frame renderer: RenderKernel on one B200.

Mirrors the reference's RenderKernel (src/kernel.h:11-59):
    Initialize(scene, ..., scattevs, sigma_s, sigma_a, tilex, tiley, w, h)
        -> Renderer(device).upload(octree) + set_params(RenderSettings)
    Render(x0, y0, tilew, tileh, samples) -> render_tile(...): sums over
        `samples` path samples per pixel, sun buffer (phb[0]) and sky buffer
        (phb[1]) as float4 tiles.
All work runs in the native library on the GPU; there is no host fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .scene import Octree
from .sky import SkyState


@dataclass
class PhaseTable:
    """Tabulated RGB phase function: pdf and CDF over the scattering angle,
    index 0 = backscatter (the layout of src/KernelSampler.cpp:8-141)."""

    pdf: np.ndarray  # (n, 3) float32
    cdf: np.ndarray  # (n, 3) float32

    @staticmethod
    def load(path: str) -> "PhaseTable":
        z = np.load(path)
        return PhaseTable(np.ascontiguousarray(z["pdf"], np.float32), np.ascontiguousarray(z["cdf"], np.float32))


@dataclass
class RenderSettings:
    sigma_s: float
    sigma_a: float
    scattevs: int
    sun_dir: np.ndarray
    sun_color: np.ndarray
    sun_angle: float
    sky: SkyState
    phase: PhaseTable
    viewi: np.ndarray
    proji: np.ndarray
    w: int
    h: int
    depth: np.ndarray | None = None   # depth texture: distance along each camera ray (shadow pass, compositing)
    depthcomp: bool = False           # KERNEL_DEPTHCOMP: camera rays stop at the depth texture
    finite_paths: bool = False        # a path sample with a non-finite sum adds nothing (DR_KERNEL_FINITE_PATHS)
    embree: bool = False              # the reference's USE_EMBREE build: occluder and depth masks (DR_KERNEL_EMBREE)
    phase_mode: int = N.DR_PHASE_MIE_REFERENCE  # DR_PHASE_MIE_REFERENCE / _MIE_EXACT / _HG
    hg_g: float = 0.0                 # DR_PHASE_HG: anisotropy (blcloudsampling.phasea)
    env_mode: int = N.DR_ENV_HOSEK    # DR_ENV_HOSEK (sky state), DR_ENV_NONE, DR_ENV_MAP
    env_map: np.ndarray | None = None  # DR_ENV_MAP: (h, w, 4) RGBA texels, row-major as MapEnv stores them
    _keep: list = field(default_factory=list, repr=False)

    def to_c(self) -> N.DrRenderParams:
        p = N.DrRenderParams()
        p.sigma_s, p.sigma_a, p.scattevs = float(self.sigma_s), float(self.sigma_a), int(self.scattevs)
        p.sun_dir[:] = [float(v) for v in np.asarray(self.sun_dir, np.float32)]
        p.sun_color[:] = [float(v) for v in np.asarray(self.sun_color, np.float32)]
        p.sun_angle = float(self.sun_angle)
        for i in range(3):
            p.sky_configs[i][:] = [float(v) for v in self.sky.configs[i]]
        p.sky_radiances[:] = [float(v) for v in self.sky.radiances]
        self._keep = []
        if self.phase is not None:
            pdf = np.ascontiguousarray(self.phase.pdf, np.float32)
            cdf = np.ascontiguousarray(self.phase.cdf, np.float32)
            self._keep = [pdf, cdf]
            p.mie_pdf, p.mie_cdf, p.mie_n = pdf.ctypes.data, cdf.ctypes.data, len(pdf)
        p.phase_mode = int(self.phase_mode)
        p.hg_g = float(self.hg_g)
        p.env_mode = int(self.env_mode)
        if self.env_mode == N.DR_ENV_MAP:
            e = np.ascontiguousarray(self.env_map, np.float32)
            if e.ndim != 3 or e.shape[2] != 4:
                raise ValueError("env_map must be (h, w, 4)")
            self._keep.append(e)
            p.env_map, p.env_h, p.env_w = e.ctypes.data, e.shape[0], e.shape[1]
        p.viewi[:] = [float(v) for v in np.asarray(self.viewi, np.float32).ravel()]
        p.proji[:] = [float(v) for v in np.asarray(self.proji, np.float32).ravel()]
        p.w, p.h = int(self.w), int(self.h)
        if self.depth is not None:
            d = np.ascontiguousarray(self.depth, np.float32).reshape(-1)
            if d.size != self.w * self.h:
                raise ValueError("depth must hold w*h values")
            self._keep.append(d)
            p.depth = d.ctypes.data
        else:
            p.depth = None
        p.flags = ((N.DR_KERNEL_DEPTHCOMP if self.depthcomp else 0) | (N.DR_KERNEL_FINITE_PATHS if self.finite_paths else 0)
                   | (N.DR_KERNEL_EMBREE if self.embree else 0))
        return p


CUDA_STREAM_LEGACY = 1  # cudaStreamLegacy: the legacy default stream as a stream handle


SURFACE_HOLDOUT = 0x2       # SCENEOBJ_HOLDOUT
OCCLUDE_ALL_SURFACES = 0    # the reference: every surface occludes
OCCLUDE_HOLDOUT_ONLY = 1    # only holdout surfaces occlude


def _surfaces(surfaces):
    keep = []
    arr = (N.DrSurface * max(len(surfaces), 1))()
    for i, (v, ix, flags) in enumerate(surfaces):
        v = np.ascontiguousarray(v, np.float32).reshape(-1, 3)
        ix = np.ascontiguousarray(ix, np.uint32).reshape(-1, 3)
        keep += [v, ix]
        arr[i] = N.DrSurface(v.ctypes.data, len(v), ix.ctypes.data, len(ix), int(flags))
    return arr, keep


def build_occluder_bvh(surfaces, mode: int = OCCLUDE_ALL_SURFACES):
    """The occluder BVH the library builds: (nodes (n, 16) float32 with the
    last four words uint32 bits, triangles (m, 12), source (m,))."""
    arr, keep = _surfaces(surfaces)
    nn, nt = C.c_uint32(0), C.c_uint32(0)
    N.check(N.lib().dr_build_occluder_bvh(arr, len(keep) // 2, mode, None, C.byref(nn), None, None, C.byref(nt)))
    nodes = np.zeros((nn.value, 16), np.float32)
    tris = np.zeros((nt.value, 12), np.float32)
    src = np.zeros(nt.value, np.uint32)
    N.check(N.lib().dr_build_occluder_bvh(arr, len(keep) // 2, mode, nodes.ctypes.data, C.byref(nn),
                                          tris.ctypes.data, src.ctypes.data, C.byref(nt)))
    return nodes, tris, src


def stream_handle(torch_stream) -> int:
    """The C-ABI handle of a torch stream.  torch's default stream reports handle 0,
    which the library reads as "the context's own stream"; it is the legacy
    default stream, so it is passed as cudaStreamLegacy instead."""
    return int(torch_stream.cuda_stream) or CUDA_STREAM_LEGACY


class Renderer:
    def __init__(self, device: int = 0):
        self._ctx = C.c_void_p()
        N.check(N.lib().dr_create(int(device), C.byref(self._ctx)))
        self.device = device
        self.sample_base = 0

    @property
    def handle(self) -> C.c_void_p:
        return self._ctx

    def close(self):
        if self._ctx:
            N.lib().dr_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def upload(self, oc: Octree):
        nodes = np.ascontiguousarray(oc.nodes)
        bricks = np.ascontiguousarray(oc.bricks, np.float32)
        d = N.DrSceneDesc(nodes.ctypes.data, len(nodes), bricks.ctypes.data, len(bricks), 8)
        sdf = getattr(oc, "sdf_bricks", None)
        if sdf is not None:
            sdf = np.ascontiguousarray(sdf, np.float32).reshape(-1, 512)
            d.sdf_bricks, d.n_sdf_leaves = sdf.ctypes.data, len(sdf)
        N.check(N.lib().dr_upload_scene(self._ctx, C.byref(d)))

    def set_occluders(self, surfaces, mode: int = OCCLUDE_ALL_SURFACES):
        """Occluder meshes (SceneOcclusion): surfaces = [(vertices (n, 3), indices
        (m, 3), flags)], flags & SURFACE_HOLDOUT marks a holdout mesh; an empty
        list removes them.  They act when the settings have embree=True."""
        arr, keep = _surfaces(surfaces)
        N.check(N.lib().dr_set_occluders(self._ctx, arr, len(keep) // 2, mode))

    def set_params(self, s: RenderSettings):
        p = s.to_c()
        N.check(N.lib().dr_set_params(self._ctx, C.byref(p)))
        self.settings = s

    def render_tile(self, x0: int, y0: int, tw: int, th: int, spp: int, seed: int = 0, sample_base: int | None = None,
                    out: tuple | None = None):
        """Sums over `spp` samples: (sun, sky) arrays of shape (th, tw, 4).  Without an
        explicit sample_base each call continues the stream (new, independent samples).
        `out` = (sun, sky) reuses caller-owned C-contiguous float32 arrays."""
        base = self.sample_base if sample_base is None else int(sample_base)
        if out is not None:
            sun, sky = out
            for a in (sun, sky):
                if a.dtype != np.float32 or a.shape != (th, tw, 4) or not a.flags.c_contiguous:
                    raise ValueError("out arrays must be C-contiguous float32 of shape (th, tw, 4)")
        else:
            sun = np.zeros((th, tw, 4), np.float32)
            sky = np.zeros((th, tw, 4), np.float32)
        rc = N.lib().dr_render_tile(self._ctx, x0, y0, tw, th, spp, int(seed), base, sun.ctypes.data,
                                    sky.ctypes.data)
        if sample_base is None and rc in (N.DR_OK, N.DR_ERR_GAVE_UP):
            self.sample_base += spp
        try:
            N.check(rc)
        except N.DrGaveUp as e:
            e.result = (sun, sky)  # written, but with some paths cut short
            raise
        return sun, sky

    def render_shadow_tile(self, x0: int, y0: int, tw: int, th: int, spp: int, seed: int = 0,
                           sample_base: int | None = None):
        """Shadow pass (RenderKernel::Shadow): per pixel the sum over `spp` sun-cone
        samples of the shadow-segment result, shape (th, tw, 4); alpha is +inf as in
        the reference.  Returns (shadow, zeros): the reference writes phb[0] only."""
        base = self.sample_base if sample_base is None else int(sample_base)
        out = np.zeros((th, tw, 4), np.float32)
        rc = N.lib().dr_shadow_tile(self._ctx, x0, y0, tw, th, spp, int(seed), base, out.ctypes.data)
        if sample_base is None and rc in (N.DR_OK, N.DR_ERR_GAVE_UP):
            self.sample_base += spp
        try:
            N.check(rc)
        except N.DrGaveUp as e:
            e.result = (out, np.zeros_like(out))
            raise
        return out, np.zeros_like(out)

    def shadow_tile_async(self, x0, y0, tw, th, spp, seed, sample_base, out_dev_ptr: int, stream_ptr: int = 0):
        N.check(N.lib().dr_shadow_tile_async(self._ctx, x0, y0, tw, th, spp, int(seed), int(sample_base),
                                             C.c_void_p(out_dev_ptr), C.c_void_p(stream_ptr) if stream_ptr else None))

    def render_tile_async(self, x0, y0, tw, th, spp, seed, sample_base, sun_dev_ptr: int, sky_dev_ptr: int,
                          stream_ptr: int = 0):
        N.check(N.lib().dr_render_tile_async(self._ctx, x0, y0, tw, th, spp, int(seed), int(sample_base),
                                             C.c_void_p(sun_dev_ptr), C.c_void_p(sky_dev_ptr),
                                             C.c_void_p(stream_ptr) if stream_ptr else None))

    def synchronize(self):
        N.check(N.lib().dr_synchronize(self._ctx))

    def check_complete(self, stream_ptr: int = 0):
        """Waits for the stream (0: the context's) and raises DrGaveUp if paths of
        the asynchronous calls since the last check were cut short."""
        N.check(N.lib().dr_check_complete(self._ctx, C.c_void_p(stream_ptr) if stream_ptr else None))

    def set_step_budget(self, steps: int = 0):
        """Tracking steps a path segment may take before it gives up (0: 2^24)."""
        N.check(N.lib().dr_set_step_budget(self._ctx, int(steps)))

    def set_camera_lists(self, pool_entries: int = 0):
        """Entries per camera leaf list pool (0: the default 2^23; N.DR_NONE: no
        lists).  Results and counters do not depend on it."""
        N.check(N.lib().dr_set_camera_lists(self._ctx, int(pool_entries)))

    def set_tuning(self, kernel: int = 0, blocks_per_sm: int = 0, event_batch: int = 0, traversal: int = 0,
                   tile: int = 0, visits: int = 0, steps: int = 0):
        t = N.DrTuning(int(kernel), int(blocks_per_sm), int(event_batch), int(traversal), int(tile), int(visits),
                       int(steps))
        N.check(N.lib().dr_set_tuning(self._ctx, C.byref(t)))

    def get_tuning(self):
        t = N.DrTuning()
        N.check(N.lib().dr_get_tuning(self._ctx, C.byref(t)))
        return (int(t.kernel), int(t.blocks_per_sm), int(t.event_batch), int(t.traversal), int(t.tile),
                int(t.visits), int(t.steps))

    # ---- differentiable rendering -------------------------------------------------
    def set_bricks_dev(self, bricks_ptr: int, n_leaves: int, majorant_scale: float = 1.0, stream_ptr: int = 0):
        """Replaces the brick pool with a device array (n_leaves x 512 float32)."""
        N.check(N.lib().dr_set_bricks_dev(self._ctx, C.c_void_p(bricks_ptr), int(n_leaves), float(majorant_scale),
                                          C.c_void_p(stream_ptr) if stream_ptr else None))

    def majorants(self, n_nodes: int) -> np.ndarray:
        out = np.zeros(n_nodes, np.float32)
        N.check(N.lib().dr_get_majorants(self._ctx, out.ctypes.data))
        return out

    def adjoint_tile_async(self, x0, y0, tw, th, spp, seed, sample_base, dsun_ptr: int, dsky_ptr: int, grad_ptr: int,
                           galb_ptr: int, stream_ptr: int = 0):
        N.check(N.lib().dr_adjoint_tile_async(self._ctx, x0, y0, tw, th, spp, int(seed), int(sample_base),
                                              C.c_void_p(dsun_ptr), C.c_void_p(dsky_ptr), C.c_void_p(grad_ptr),
                                              C.c_void_p(galb_ptr), C.c_void_p(stream_ptr) if stream_ptr else None))

    def reweighted_loss_async(self, x0, y0, tw, th, spp, seed, sample_base, dsun_ptr: int, dsky_ptr: int,
                              pert_ptr: int, loss_ptr: int, stream_ptr: int = 0):
        """Adds to the double at loss_ptr the linearised loss of the tile's paths
        replayed with decisions from the uploaded bricks, each weighted by its
        probability ratio under the bricks at pert_ptr (the adjoint's
        finite-difference check)."""
        N.check(N.lib().dr_reweighted_loss_async(self._ctx, x0, y0, tw, th, spp, int(seed), int(sample_base),
                                                 C.c_void_p(dsun_ptr), C.c_void_p(dsky_ptr), C.c_void_p(pert_ptr),
                                                 C.c_void_p(loss_ptr), C.c_void_p(stream_ptr) if stream_ptr else None))

    def adjoint_transmittance(self, ro, rd, weights, nsamp: int, seed: int, n_leaves: int):
        """(d sum_r w_r T_r / d brick samples (n_leaves, 512), T per ray) on the GPU."""
        ro = np.ascontiguousarray(ro, np.float32).reshape(-1)
        rd = np.ascontiguousarray(rd, np.float32).reshape(-1)
        w = np.ascontiguousarray(weights, np.float32).reshape(-1)
        grad = np.zeros(n_leaves * 512, np.float32)
        T = np.zeros(len(w), np.float64)
        N.check(N.lib().dr_adjoint_transmittance(self._ctx, ro.ctypes.data, rd.ctypes.data, w.ctypes.data, len(w),
                                                 int(nsamp), int(seed), grad.ctypes.data, T.ctypes.data))
        return grad.reshape(n_leaves, 512), T

    def counters(self) -> dict:
        c = N.DrCounters()
        N.check(N.lib().dr_get_counters(self._ctx, C.byref(c)))
        return c.as_dict()

    def reset_counters(self):
        N.check(N.lib().dr_reset_counters(self._ctx))

    # ---- parity probes ---------------------------------------------------------
    def probe_leaf_sequence(self, ro, rd, maxn: int = 256):
        ro = np.ascontiguousarray(ro, np.float32).reshape(-1, 3)
        rd = np.ascontiguousarray(rd, np.float32).reshape(-1, 3)
        n = len(ro)
        nodes = np.zeros((n, maxn), np.uint32)
        a = np.zeros((n, maxn), np.float32)
        b = np.zeros((n, maxn), np.float32)
        cnt = np.zeros(n, np.uint32)
        N.check(N.lib().dr_probe_leaf_sequence(self._ctx, ro.ctypes.data, rd.ctypes.data, n, maxn, nodes.ctypes.data,
                                               a.ctypes.data, b.ctypes.data, cnt.ctypes.data))
        return nodes, a, b, cnt

    def probe_occlusion(self, ro, rd) -> np.ndarray:
        """1 per ray that hits an occluder at t in [0, 1e6] (the GPU traversal)."""
        ro = np.ascontiguousarray(ro, np.float32).reshape(-1, 3)
        rd = np.ascontiguousarray(rd, np.float32).reshape(-1, 3)
        hit = np.zeros(len(ro), np.uint32)
        N.check(N.lib().dr_probe_occlusion(self._ctx, ro.ctypes.data, rd.ctypes.data, len(ro), hit.ctypes.data))
        return hit

    def probe_density(self, leaf_nodes, points):
        leaf_nodes = np.ascontiguousarray(leaf_nodes, np.uint32)
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        out = np.zeros(len(pts), np.float32)
        N.check(N.lib().dr_probe_density(self._ctx, leaf_nodes.ctypes.data, pts.ctypes.data, len(pts),
                                         out.ctypes.data))
        return out

    def probe_paths(self, px, py, sample, seed: int):
        px = np.ascontiguousarray(px, np.uint32)
        py = np.ascontiguousarray(py, np.uint32)
        sm = np.ascontiguousarray(sample, np.uint64)
        n = len(px)
        a = np.zeros((n, 4), np.float32)
        b = np.zeros((n, 4), np.float32)
        N.check(N.lib().dr_probe_paths(self._ctx, px.ctypes.data, py.ctypes.data, sm.ctypes.data, n, int(seed),
                                       a.ctypes.data, b.ctypes.data))
        return a, b

    def probe_sampler(self, what: int, inputs: np.ndarray, n: int):
        x = np.ascontiguousarray(inputs, np.float32).reshape(-1)
        width = {N.DR_PROBE_MIE_THETA: 1, N.DR_PROBE_MIE_EXACT_DIR: 2, N.DR_PROBE_HG_EVAL: 1}.get(what, 3)
        out = np.zeros(width * n, np.float32)
        N.check(N.lib().dr_probe_sampler(self._ctx, int(what), x.ctypes.data, int(n), out.ctypes.data))
        return out if width == 1 else out.reshape(n, width)

    def probe_transmittance(self, ro, rd, nsamp: int, seed: int = 0):
        ro = np.ascontiguousarray(ro, np.float32).reshape(-1, 3)
        rd = np.ascontiguousarray(rd, np.float32).reshape(-1, 3)
        out = np.zeros(len(ro), np.float64)
        N.check(N.lib().dr_probe_transmittance(self._ctx, ro.ctypes.data, rd.ctypes.data, len(ro), int(nsamp),
                                               int(seed), out.ctypes.data))
        return out


@dataclass
class BatchView:
    """One view of a batch: scene index, settings, region, samples per launch, seed."""
    scene: int
    settings: RenderSettings
    spp: int
    seed: int = 0
    region: tuple | None = None   # (x0, y0, tw, th); None = the whole image


class Batch:
    """Many scenes and views rendered by one launch of a CUDA graph (dr_batch_*):
    a persistent kernel over the views, large views optionally in kernels of
    their own (set_split).  Launch k renders samples [k spp, (k+1) spp) of each
    view, the streams Renderer.render_tile draws with sample_base = k spp."""

    SPLIT_AUTO = (1 << 64) - 1  # DR_BATCH_SPLIT_AUTO

    def __init__(self, renderer: "Renderer", scenes: list, views: list):
        descs = (N.DrSceneDesc * len(scenes))()
        self._keep = []
        for i, oc in enumerate(scenes):
            nodes = np.ascontiguousarray(oc.nodes)
            bricks = np.ascontiguousarray(oc.bricks, np.float32)
            self._keep += [nodes, bricks]
            descs[i] = N.DrSceneDesc(nodes.ctypes.data, len(nodes), bricks.ctypes.data, len(bricks), 8)
            sdf = getattr(oc, "sdf_bricks", None)
            if sdf is not None:
                sdf = np.ascontiguousarray(sdf, np.float32).reshape(-1, 512)
                self._keep.append(sdf)
                descs[i].sdf_bricks, descs[i].n_sdf_leaves = sdf.ctypes.data, len(sdf)
        bv = (N.DrBatchView * len(views))()
        params = []
        self.views = list(views)
        for i, v in enumerate(views):
            p = v.settings.to_c()
            params.append(p)
            x0, y0, tw, th = v.region if v.region is not None else (0, 0, v.settings.w, v.settings.h)
            bv[i] = N.DrBatchView(int(v.scene), C.cast(C.pointer(p), C.c_void_p), x0, y0, tw, th, int(v.spp),
                                  int(v.seed))
        self.regions = [v.region if v.region is not None else (0, 0, v.settings.w, v.settings.h) for v in views]
        self._h = C.c_void_p()
        self.renderer = renderer
        N.check(N.lib().dr_batch_create(renderer.handle, descs, len(scenes), bv, len(views), C.byref(self._h)))

    def close(self):
        if self._h:
            N.lib().dr_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_tuning(self, kernel: int = 0, blocks_per_sm: int = 0, event_batch: int = 0, traversal: int = 0,
                   tile: int = 0, visits: int = 0, steps: int = 0):
        t = N.DrTuning(0, int(blocks_per_sm), int(event_batch), int(traversal), int(tile), int(visits), int(steps))
        N.check(N.lib().dr_batch_set_tuning(self._h, C.byref(t)))

    def get_tuning(self):
        t = N.DrTuning()
        N.check(N.lib().dr_batch_get_tuning(self._h, C.byref(t)))
        return (int(t.kernel), int(t.blocks_per_sm), int(t.event_batch), int(t.traversal), int(t.tile),
                int(t.visits), int(t.steps))

    def launch(self, stream_ptr: int = 0):
        N.check(N.lib().dr_batch_launch(self._h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def output_ptrs(self, view: int):
        a, b = C.c_void_p(), C.c_void_p()
        N.check(N.lib().dr_batch_output(self._h, int(view), C.byref(a), C.byref(b)))
        return a.value, b.value

    def read(self, view: int):
        """(sun, sky) sums of the last launch for one view, shape (th, tw, 4)."""
        _, _, tw, th = self.regions[view]
        sun = np.zeros((th, tw, 4), np.float32)
        sky = np.zeros((th, tw, 4), np.float32)
        N.check(N.lib().dr_batch_read(self._h, int(view), sun.ctypes.data, sky.ctypes.data))
        return sun, sky

    def info(self):
        n, k = C.c_uint64(), C.c_uint64()
        N.check(N.lib().dr_batch_info(self._h, C.byref(n), C.byref(k)))
        return int(n.value), int(k.value)

    def set_split(self, min_paths: int):
        """Views of at least min_paths paths per launch get a kernel of their own
        (0: one batched kernel for every view; SPLIT_AUTO: the library's rule)."""
        N.check(N.lib().dr_batch_set_split(self._h, int(min_paths)))

    def get_split(self):
        """(min_paths setting, views with a kernel of their own in the graph)."""
        m, k = C.c_uint64(), C.c_uint32()
        N.check(N.lib().dr_batch_get_split(self._h, C.byref(m), C.byref(k)))
        return int(m.value), int(k.value)
