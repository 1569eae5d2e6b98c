"""ctypes access to the two CPU checkers (TEST INFRASTRUCTURE ONLY)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libdroplet_ref.so")
REF_ENV_LIB = os.path.join(HERE, "_ref", "libdroplet_ref_env.so")  # built without USE_ARHOSEK_SKYMODEL
PORT_LIB = os.path.join(HERE, "_port", "liboracle_port.so")
NODE_DTYPE = np.dtype([("ce", "<f4", 4), ("chn", "<u4", 8), ("volx", "<u4", 2), ("qval", "<f4", 2)])
assert NODE_DTYPE.itemsize == 64


def reference_src() -> str:
    """Directory of the reference's sources: $DROPLET_REFERENCE_SRC, else the
    `REF ?=` default of oracle/Makefile (the recipe that compiles them)."""
    env = os.environ.get("DROPLET_REFERENCE_SRC")
    if env:
        return env
    with open(os.path.join(HERE, "Makefile")) as f:
        for line in f:
            if line.startswith("REF") and "?=" in line:
                return line.split("?=", 1)[1].strip()
    raise RuntimeError("oracle/Makefile has no REF default")


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def port_available() -> bool:
    return os.path.exists(PORT_LIB)


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class OrcParams(C.Structure):
    _fields_ = [
        ("sigma_s", C.c_float), ("sigma_a", C.c_float), ("scattevs", C.c_uint32),
        ("sun_dir", C.c_float * 3), ("sun_color", C.c_float * 3), ("sun_cos_angle", C.c_float),
        ("sky_cfg", (C.c_float * 9) * 3), ("sky_rad", C.c_float * 3),
        ("mie_pdf", C.c_void_p), ("mie_cdf", C.c_void_p), ("mie_n", C.c_uint32),
        ("viewi", C.c_float * 16), ("proji", C.c_float * 16), ("w", C.c_uint32), ("h", C.c_uint32),
        ("depth", C.c_float), ("depth_map", C.c_void_p), ("depthcomp", C.c_uint32),
        ("phase_mode", C.c_uint32), ("mie_exact", C.c_void_p), ("finite_paths", C.c_uint32),
        ("embree", C.c_uint32), ("hg_g", C.c_float), ("env_mode", C.c_uint32), ("env_map", C.c_void_p),
        ("env_w", C.c_uint32), ("env_h", C.c_uint32),
    ]


class OrcScene(C.Structure):
    _fields_ = [("nodes", C.c_void_p), ("n_nodes", C.c_uint32), ("bricks", C.c_void_p), ("n_leaves", C.c_uint32),
                ("lvoxc", C.c_uint32), ("occ_tris", C.c_void_p), ("occ_n", C.c_uint32), ("sdf_bricks", C.c_void_p)]


class OrcCounters(C.Structure):
    _fields_ = [("vertices", C.c_uint64), ("node_visits", C.c_uint64), ("density_lookups", C.c_uint64),
                ("mie_evals", C.c_uint64), ("paths", C.c_uint64)]

    def as_dict(self):
        return {f: int(getattr(self, f)) for f, _ in self._fields_}


class Port:
    """The C restatement (oracle/port)."""

    def __init__(self, path: str = PORT_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle port not built: {path} (make -C oracle port)")
        L = C.CDLL(path)
        vp, u32, f32 = C.c_void_p, C.c_uint32, C.c_float
        L.orc_build_octree.argtypes = [vp, vp, u32, f32, u32, C.POINTER(vp), C.POINTER(u32), C.POINTER(vp),
                                       C.POINTER(u32), C.POINTER(u32), C.POINTER(u32)]
        L.orc_build_octree.restype = C.c_int
        L.orc_free.argtypes = [vp]
        L.orc_leaf_sequence.argtypes = [vp, vp, vp, u32, vp, vp, vp]
        L.orc_leaf_sequence.restype = u32
        L.orc_point_lookup.argtypes = [vp, vp, C.POINTER(C.c_int)]
        L.orc_point_lookup.restype = u32
        L.orc_sample_voxel_space.argtypes = [vp, vp, vp, u32]
        L.orc_sample_voxel_space.restype = f32
        L.orc_mie_eval_rgb.argtypes = [C.POINTER(OrcParams), f32, vp]
        L.orc_mie_sample_theta_scan.argtypes = [C.POINTER(OrcParams), f32]
        L.orc_mie_sample_theta_scan.restype = f32
        L.orc_mie_sample_theta_bisect.argtypes = [C.POINTER(OrcParams), f32]
        L.orc_mie_sample_theta_bisect.restype = f32
        L.orc_mie_sample.argtypes = [C.POINTER(OrcParams), vp, f32, f32, vp]
        L.orc_sun_sample.argtypes = [C.POINTER(OrcParams), f32, f32, vp]
        L.orc_sky_eval.argtypes = [C.POINTER(OrcParams), vp, vp]
        L.orc_camera_ray.argtypes = [C.POINTER(OrcParams), u32, u32, vp, vp, C.POINTER(C.c_int)]
        L.orc_optical_depth.argtypes = [C.POINTER(OrcScene), vp, vp, C.c_double]
        L.orc_optical_depth.restype = C.c_double
        L.orc_optical_depth_grad.argtypes = [C.POINTER(OrcScene), vp, vp, C.c_double, vp]
        L.orc_single_scatter_sun.argtypes = [C.POINTER(OrcScene), C.POINTER(OrcParams), vp, vp, C.c_uint32, C.c_double,
                                             C.c_uint32, C.c_uint32, vp, vp, vp]
        L.orc_sun_hit_fraction.argtypes = [C.POINTER(OrcParams), C.c_uint32, C.c_uint32]
        L.orc_sun_hit_fraction.restype = C.c_double
        L.orc_math_eval.argtypes = [C.c_int, vp, C.c_uint32, vp]
        L.orc_render_tile_mt.argtypes = [C.POINTER(OrcScene), C.POINTER(OrcParams), u32, u32, u32, u32, u32,
                                         C.c_uint64, C.c_uint64, vp, vp, C.POINTER(OrcCounters), C.c_int]
        L.orc_render_tile_mt.restype = C.c_int
        L.orc_adjoint_tile_mt.argtypes = [C.POINTER(OrcScene), C.POINTER(OrcParams), u32, u32, u32, u32, u32,
                                          C.c_uint64, C.c_uint64, vp, vp, vp, vp, C.c_int]
        L.orc_adjoint_tile_mt.restype = C.c_int
        L.orc_hg_eval.argtypes = [f32, f32]
        L.orc_hg_eval.restype = f32
        L.orc_hg_sample.argtypes = [f32, vp, f32, f32, vp]
        L.orc_atan2_ref.argtypes = [f32, f32]
        L.orc_atan2_ref.restype = f32
        L.orc_env_map_eval.argtypes = [C.POINTER(OrcParams), vp, vp]
        L.orc_sky_light.argtypes = [C.POINTER(OrcParams), vp, vp]
        L.orc_occluded.argtypes = [C.POINTER(OrcScene), vp, vp]
        L.orc_occluded.restype = C.c_int
        L.orc_shadow_ray.argtypes = [C.POINTER(OrcParams), u32, u32, C.c_uint64, C.c_uint64, vp, vp]
        L.orc_shadow_ray.restype = C.c_int
        L.orc_occluded_fp64.argtypes = [C.POINTER(OrcScene), vp, vp, C.POINTER(C.c_double)]
        L.orc_occluded_fp64.restype = C.c_int
        L.orc_reweighted_loss.argtypes = [C.POINTER(OrcScene), C.POINTER(OrcParams), u32, u32, u32, u32, u32,
                                          C.c_uint64, C.c_uint64, vp, vp, vp]
        L.orc_reweighted_loss.restype = C.c_double
        L.orc_adjoint_transmittance.argtypes = [C.POINTER(OrcScene), C.POINTER(OrcParams), vp, vp, vp, u32,
                                                C.c_uint64, C.c_uint64, vp, vp]
        L.orc_mie_exact_table.argtypes = [vp, u32, vp]
        L.orc_mie_exact_dirs.argtypes = [vp, u32, vp, u32, vp, vp]
        L.orc_shadow_tile_mt.argtypes = [C.POINTER(OrcScene), C.POINTER(OrcParams), u32, u32, u32, u32, u32,
                                         C.c_uint64, C.c_uint64, vp, C.POINTER(OrcCounters), C.c_int]
        L.orc_shadow_tile_mt.restype = C.c_int
        L.orc_render_path.argtypes = [C.POINTER(OrcScene), C.POINTER(OrcParams), u32, u32, C.c_uint64, C.c_uint64,
                                      vp, vp, C.POINTER(OrcCounters)]
        L.orc_transmittance_mc.argtypes = [C.POINTER(OrcScene), C.POINTER(OrcParams), vp, vp, C.c_uint64, C.c_uint64]
        L.orc_transmittance_mc.restype = C.c_double
        self.L = L

    # -- scene build -------------------------------------------------------------
    def build_octree(self, block_origin: np.ndarray, block_values: np.ndarray, voxel_size: float, maxdepth: int = 12):
        org = np.ascontiguousarray(block_origin, np.int32)
        vals = np.ascontiguousarray(block_values, np.float32)
        pn, pb = C.c_void_p(), C.c_void_p()
        nn, nl, lv, ml = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
        rc = self.L.orc_build_octree(_p(org), _p(vals), len(org), voxel_size, maxdepth, C.byref(pn), C.byref(nn),
                                     C.byref(pb), C.byref(nl), C.byref(lv), C.byref(ml))
        if rc != 0:
            raise ValueError(f"orc_build_octree failed ({rc})")
        nodes = np.frombuffer(C.string_at(pn, nn.value * 64), NODE_DTYPE).copy()
        bricks = np.frombuffer(C.string_at(pb, nl.value * lv.value ** 3 * 4), np.float32).copy()
        self.L.orc_free(pn)
        self.L.orc_free(pb)
        return nodes, bricks.reshape(nl.value, lv.value ** 3), int(ml.value)

    @staticmethod
    def scene(nodes: np.ndarray, bricks: np.ndarray, occ: np.ndarray = None, sdf: np.ndarray = None) -> OrcScene:
        """occ: occluder triangles from occluder_triangles(); sdf: the surface brick
        pool (float32, 512 per brick); both kept alive by the caller."""
        S = OrcScene(nodes.ctypes.data, len(nodes), bricks.ctypes.data, len(bricks), 8)
        if occ is not None and len(occ):
            assert occ.dtype == np.float32 and occ.flags.c_contiguous and occ.shape[1] == 12
            S.occ_tris, S.occ_n = occ.ctypes.data, len(occ)
        if sdf is not None:
            assert sdf.dtype == np.float32 and sdf.flags.c_contiguous
            S.sdf_bricks = sdf.ctypes.data
        return S

    @staticmethod
    def occluder_triangles(surfaces, mode: int = 0) -> np.ndarray:
        """Occluder triangles of SceneOcclusion::Initialize (src/SceneOcclusion.cpp:19-56)
        in surface order, 12 floats each (v0, e1 = v1 - v0, e2 = v2 - v0; w 0).
        surfaces: (vertices (n, 3), indices (m, 3), flags); mode 0 = every
        surface (the reference's `!flags & SCENEOBJ_HOLDOUT` is always 0),
        1 = only surfaces with flags & 2 (SCENEOBJ_HOLDOUT)."""
        out = []
        for v, ix, flags in surfaces:
            if mode == 1 and not (flags & 2):
                continue
            v = np.asarray(v, np.float32).reshape(-1, 3)
            ix = np.asarray(ix, np.int64).reshape(-1, 3)
            t = np.zeros((len(ix), 12), np.float32)
            v0, v1, v2 = v[ix[:, 0]], v[ix[:, 1]], v[ix[:, 2]]
            t[:, 0:3], t[:, 4:7], t[:, 8:11] = v0, v1 - v0, v2 - v0
            out.append(t)
        return np.ascontiguousarray(np.concatenate(out) if out else np.zeros((0, 12), np.float32))

    def hg_eval(self, g, ct):
        return np.array([self.L.orc_hg_eval(g, float(c)) for c in np.asarray(ct, np.float32)], np.float32)

    def hg_sample(self, g, iv, u1, u2):
        iv = np.ascontiguousarray(iv, np.float32).reshape(-1, 3)
        out = np.zeros_like(iv)
        for i in range(len(iv)):
            self.L.orc_hg_sample(g, _p(iv[i]), float(u1[i]), float(u2[i]), _p(out[i]))
        return out

    def atan2_ref(self, y, x):
        return np.array([self.L.orc_atan2_ref(float(a), float(b)) for a, b in zip(y, x)], np.float32)

    def env_map_eval(self, P, rd):
        rd = np.ascontiguousarray(rd, np.float32).reshape(-1, 3)
        out = np.zeros_like(rd)
        for i in range(len(rd)):
            self.L.orc_env_map_eval(C.byref(P), _p(rd[i]), _p(out[i]))
        return out

    def sky_light(self, P, rd):
        rd = np.ascontiguousarray(rd, np.float32).reshape(-1, 3)
        out = np.zeros_like(rd)
        for i in range(len(rd)):
            self.L.orc_sky_light(C.byref(P), _p(rd[i]), _p(out[i]))
        return out

    def occluded(self, S, ro, rd) -> np.ndarray:
        """Binary32 any-hit answer per ray (the GPU's triangle test, every triangle)."""
        ro = np.ascontiguousarray(ro, np.float32).reshape(-1, 3)
        rd = np.ascontiguousarray(rd, np.float32).reshape(-1, 3)
        return np.array([self.L.orc_occluded(C.byref(S), _p(ro[i]), _p(rd[i])) for i in range(len(ro))], np.uint32)

    def shadow_rays(self, P, x0, y0, tw, th, spp, seed, sample_base=0):
        """(origins, directions, active) of the shadow pass's segments over a tile,
        in (row, column, sample) order."""
        n = th * tw * spp
        ro = np.zeros((n, 3), np.float32)
        rd = np.zeros((n, 3), np.float32)
        act = np.zeros(n, bool)
        k = 0
        for j in range(th):
            for i in range(tw):
                for s in range(spp):
                    act[k] = self.L.orc_shadow_ray(C.byref(P), x0 + i, y0 + j, seed, sample_base + s, _p(ro[k]),
                                                   _p(rd[k]))
                    k += 1
        return ro, rd, act

    def occluded_fp64(self, S, ro, rd):
        """(hit, edge margin) per ray of the FP64 test."""
        ro = np.ascontiguousarray(ro, np.float64).reshape(-1, 3)
        rd = np.ascontiguousarray(rd, np.float64).reshape(-1, 3)
        hit = np.zeros(len(ro), np.uint32)
        marg = np.zeros(len(ro))
        m = C.c_double()
        for i in range(len(ro)):
            hit[i] = self.L.orc_occluded_fp64(C.byref(S), _p(ro[i]), _p(rd[i]), C.byref(m))
            marg[i] = m.value
        return hit, marg

    def leaf_sequence(self, nodes, ro, rd, maxn=4096):
        ro = np.ascontiguousarray(ro, np.float32)
        rd = np.ascontiguousarray(rd, np.float32)
        n_ = np.zeros(maxn, np.uint32)
        a = np.zeros(maxn, np.float32)
        b = np.zeros(maxn, np.float32)
        k = self.L.orc_leaf_sequence(_p(nodes), _p(ro), _p(rd), maxn, _p(n_), _p(a), _p(b))
        return n_[:k], a[:k], b[:k]

    def point_lookup(self, nodes, p):
        d = C.c_int()
        p = np.ascontiguousarray(p, np.float64)
        r = self.L.orc_point_lookup(_p(nodes), _p(p), C.byref(d))
        return int(r), int(d.value)

    def sample_voxel_space(self, p, brick, ce):
        p = np.ascontiguousarray(p, np.float32)
        brick = np.ascontiguousarray(brick, np.float32)
        ce = np.ascontiguousarray(ce, np.float32)
        return float(self.L.orc_sample_voxel_space(_p(p), _p(brick), _p(ce), 8))

    @staticmethod
    def params(cfg: dict, keep: list) -> OrcParams:
        """OrcParams from a render configuration dict (see tests' helpers)."""
        P = OrcParams()
        P.sigma_s, P.sigma_a, P.scattevs = cfg["sigma_s"], cfg["sigma_a"], cfg["scattevs"]
        P.sun_dir[:] = [float(v) for v in cfg["sun_dir"]]
        P.sun_color[:] = [float(v) for v in cfg["sun_color"]]
        P.sun_cos_angle = float(np.cos(np.float32(cfg["sun_angle"]), dtype=np.float32)) \
            if "sun_cos" not in cfg else float(cfg["sun_cos"])
        cfgs = np.asarray(cfg["sky_configs"], np.float64).astype(np.float32)
        for i in range(3):
            P.sky_cfg[i][:] = [float(v) for v in cfgs[i]]
        P.sky_rad[:] = [float(v) for v in np.asarray(cfg["sky_radiances"], np.float64).astype(np.float32)]
        pdf = np.ascontiguousarray(cfg["mie_pdf"], np.float32)
        cdf = np.ascontiguousarray(cfg["mie_cdf"], np.float32)
        keep += [pdf, cdf]
        P.mie_pdf, P.mie_cdf, P.mie_n = pdf.ctypes.data, cdf.ctypes.data, len(pdf)
        P.viewi[:] = [float(v) for v in cfg["viewi"]]
        P.proji[:] = [float(v) for v in cfg["proji"]]
        P.w, P.h = cfg["w"], cfg["h"]
        P.depth = float(np.finfo(np.float32).max)
        if cfg.get("depth") is not None:
            dm = np.ascontiguousarray(cfg["depth"], np.float32).reshape(-1)
            assert dm.size == cfg["w"] * cfg["h"]
            keep.append(dm)
            P.depth_map = dm.ctypes.data
            P.depthcomp = 1 if cfg.get("depthcomp") else 0
        P.finite_paths = 1 if cfg.get("finite_paths") else 0
        P.embree = 1 if cfg.get("embree") else 0
        P.hg_g = float(cfg.get("hg_g", 0.0))
        P.env_mode = int(cfg.get("env_mode", 0))
        if P.env_mode == 2:
            em = np.ascontiguousarray(cfg["env_map"], np.float32)
            keep.append(em)
            P.env_map, P.env_h, P.env_w = em.ctypes.data, em.shape[0], em.shape[1]
        if cfg.get("phase_mode", 0) == 1:
            tab = Port().mie_exact_table(pdf)
            keep.append(tab)
            P.phase_mode, P.mie_exact = 1, tab.ctypes.data
        elif cfg.get("phase_mode", 0) == 2:
            P.phase_mode = 2
        return P

    def mie_exact_table(self, pdf: np.ndarray) -> np.ndarray:
        """Exact-mode sampler table from the RGB pdf (n x 3): 8 n + 4 floats."""
        pdf = np.ascontiguousarray(pdf, np.float32)
        out = np.zeros(8 * len(pdf) + 4, np.float32)
        self.L.orc_mie_exact_table(_p(pdf), len(pdf), _p(out))
        return out

    def mie_exact_dirs(self, tab: np.ndarray, n: int, u1: np.ndarray):
        """(ct, st) of exact-mode samples for the uniforms u1."""
        u1 = np.ascontiguousarray(u1, np.float32)
        ct = np.zeros(len(u1), np.float32)
        st = np.zeros(len(u1), np.float32)
        self.L.orc_mie_exact_dirs(_p(tab), n, _p(u1), len(u1), _p(ct), _p(st))
        return ct, st

    def render_tile(self, S, P, x0, y0, tw, th, spp, seed, sample_base=0, threads=0):
        sun = np.zeros((th, tw, 4), np.float32)
        sky = np.zeros((th, tw, 4), np.float32)
        cnt = OrcCounters()
        nt = threads if threads > 0 else (os.cpu_count() or 1)
        self.L.orc_render_tile_mt(C.byref(S), C.byref(P), x0, y0, tw, th, spp, seed, sample_base, _p(sun), _p(sky),
                                  C.byref(cnt), nt)
        return sun, sky, cnt.as_dict()

    def shadow_tile(self, S, P, x0, y0, tw, th, spp, seed, sample_base=0, threads=0):
        out = np.zeros((th, tw, 4), np.float32)
        cnt = OrcCounters()
        nt = threads if threads > 0 else (os.cpu_count() or 1)
        self.L.orc_shadow_tile_mt(C.byref(S), C.byref(P), x0, y0, tw, th, spp, seed, sample_base, _p(out),
                                  C.byref(cnt), nt)
        return out, cnt.as_dict()

    def adjoint_tile(self, S, P, x0, y0, tw, th, spp, seed, sample_base, dsun, dsky, threads=0):
        """(d loss / d brick samples (n_leaves, 512) float64, d loss / d albedo) for
        dsun/dsky = dL/d(tile sums), shape (th, tw, 4)."""
        dsun = np.ascontiguousarray(dsun, np.float32)
        dsky = np.ascontiguousarray(dsky, np.float32)
        grad = np.zeros(S.n_leaves * 512, np.float64)
        galb = np.zeros(1, np.float64)
        nt = threads if threads > 0 else (os.cpu_count() or 1)
        rc = self.L.orc_adjoint_tile_mt(C.byref(S), C.byref(P), x0, y0, tw, th, spp, seed, sample_base, _p(dsun),
                                        _p(dsky), _p(grad), _p(galb), nt)
        if rc != 0:
            raise MemoryError("orc_adjoint_tile_mt")
        return grad.reshape(-1, 512), float(galb[0])

    def reweighted_loss(self, S, P, x0, y0, tw, th, spp, seed, sample_base, dsun, dsky, pert):
        """Linearised loss of the reweighted replay: decisions from the scene's
        bricks, each weighted by its probability ratio under pert (n_leaves, 512)."""
        dsun = np.ascontiguousarray(dsun, np.float32)
        dsky = np.ascontiguousarray(dsky, np.float32)
        pert = np.ascontiguousarray(pert, np.float32)
        return float(self.L.orc_reweighted_loss(C.byref(S), C.byref(P), x0, y0, tw, th, spp, seed, sample_base,
                                                _p(dsun), _p(dsky), _p(pert)))

    def adjoint_transmittance(self, S, P, ro, rd, w, nsamp, seed):
        ro = np.ascontiguousarray(ro, np.float32)
        rd = np.ascontiguousarray(rd, np.float32)
        w = np.ascontiguousarray(w, np.float32)
        grad = np.zeros(S.n_leaves * 512, np.float64)
        T = np.zeros(len(w), np.float64)
        self.L.orc_adjoint_transmittance(C.byref(S), C.byref(P), _p(ro), _p(rd), _p(w), len(w), nsamp, seed,
                                         _p(grad), _p(T))
        return grad.reshape(-1, 512), T

    def optical_depth_grad(self, S, ro, rd, tmax=1e30):
        """FP64 d(optical depth)/d(brick samples) of one ray (quadrature oracle)."""
        ro = np.ascontiguousarray(ro, np.float64)
        rd = np.ascontiguousarray(rd, np.float64)
        grad = np.zeros(S.n_leaves * 512, np.float64)
        self.L.orc_optical_depth_grad(C.byref(S), _p(ro), _p(rd), tmax, _p(grad))
        return grad.reshape(-1, 512)

    def single_scatter_sun(self, S, P, ro, rd, wc=(1.0, 1.0, 1.0), grad=True, nu=4, nphi=8, p_hit=None):
        """FP64 quadrature of the expected sun sum of one path sample per camera
        ray with scattevs = 1 (out (n, 3)), and d(sum_r sum_c wc_c out[r, c])/d
        brick sample (n_leaves, lvoxc^3) when grad (port/fp64.c)."""
        ro = np.ascontiguousarray(ro, np.float32).reshape(-1, 3)
        rd = np.ascontiguousarray(rd, np.float32).reshape(-1, 3)
        if p_hit is None:
            p_hit = self.sun_hit_fraction(P)
        out = np.zeros((len(ro), 3), np.float64)
        w = np.ascontiguousarray(wc, np.float64)
        g = np.zeros((S.n_leaves, S.lvoxc ** 3), np.float64) if grad else None
        self.L.orc_single_scatter_sun(C.byref(S), C.byref(P), _p(ro), _p(rd), len(ro), float(p_hit), nu, nphi, _p(w),
                                      _p(out), None if g is None else _p(g))
        return out, g

    def math_eval(self, kind: int, x):
        """orc_math.h's function `kind` (0 log, 1 exp, 2 sin, 3 cos, 4 x^1.5, 5 x^2.2) on float32 x."""
        x = np.ascontiguousarray(x, np.float32)
        out = np.zeros_like(x)
        self.L.orc_math_eval(int(kind), _p(x), len(x), _p(out))
        return out

    def sun_hit_fraction(self, P, n1=2048, n2=512):
        return float(self.L.orc_sun_hit_fraction(C.byref(P), n1, n2))

    def optical_depth(self, S, ro, rd, tmax=1e30):
        ro = np.ascontiguousarray(ro, np.float64)
        rd = np.ascontiguousarray(rd, np.float64)
        return float(self.L.orc_optical_depth(C.byref(S), _p(ro), _p(rd), tmax))

    def render_path(self, S, P, px, py, seed, sample):
        a = np.zeros(4, np.float32)
        b = np.zeros(4, np.float32)
        cnt = OrcCounters()
        self.L.orc_render_path(C.byref(S), C.byref(P), px, py, seed, sample, _p(a), _p(b), C.byref(cnt))
        return a, b, cnt.as_dict()


class Reference:
    """The reference's own sources compiled unmodified (oracle/_ref)."""

    def __init__(self, path: str = REF_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"reference oracle not built: {path} (make -C oracle ref)")
        L = C.CDLL(path)
        vp, u32, f32, f64 = C.c_void_p, C.c_uint32, C.c_float, C.c_double
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_scene_create.argtypes = [vp, u32, vp, u32, u32]
        L.ref_scene_create.restype = vp
        L.ref_scene_destroy.argtypes = [vp]
        L.ref_scene_create_sdf.argtypes = [vp, u32, vp, u32, vp, u32, u32]
        L.ref_scene_create_sdf.restype = vp
        L.ref_leaf_sequence.argtypes = [vp, C.c_int, vp, vp, u32, vp, vp, vp]
        L.ref_leaf_sequence.restype = u32
        L.ref_sky_state.argtypes = [f64, f64, f64, vp, vp]
        L.ref_solar_elevation.argtypes = [vp]
        L.ref_solar_elevation.restype = f32
        L.ref_render.argtypes = [vp, vp, vp, vp, vp, f32, f64, f64, u32, f32, f32, u32, u32, u32, u32, u32, u32, u32,
                                 vp, vp, vp, u32]
        L.ref_render.restype = C.c_int
        L.ref_shadow.argtypes = [vp, vp, vp, vp, vp, f32, u32, f32, f32, u32, u32, u32, u32, u32, u32, u32, vp, vp]
        L.ref_shadow.restype = C.c_int
        L.ref_sample_voxel_space.argtypes = [vp, vp, vp, u32]
        L.ref_sample_voxel_space.restype = f32
        L.ref_mie_table_size.restype = u32
        L.ref_mie_tables.argtypes = [vp, vp]
        L.ref_mie_eval.argtypes = [vp, u32, vp, vp]
        L.ref_mie_sample.argtypes = [vp, vp, vp, u32, vp]
        L.ref_sun_ops.argtypes = [vp, vp, f32, vp, vp, vp, u32, vp, vp, vp]
        L.ref_rng_draw.argtypes = [vp, u32, vp]
        L.ref_hg_eval.argtypes = [f32, vp, u32, vp]
        L.ref_hg_sample.argtypes = [f32, vp, vp, vp, u32, vp]
        L.ref_atan2.argtypes = [vp, vp, u32, vp]
        L.ref_env_eval.argtypes = [u32, u32, vp, vp, u32, vp]
        L.ref_has_hosek.restype = C.c_int
        L.ref_render_ex.argtypes = [vp, vp, vp, vp, vp, f32, f64, f64, u32, f32, f32, u32, u32, u32, u32, u32, u32,
                                    u32, vp, vp, vp, u32, C.c_int, f32, u32, u32, vp]
        L.ref_render_ex.restype = C.c_int
        self.L = L

    def hg_eval(self, g, ct):
        ct = np.ascontiguousarray(ct, np.float32)
        out = np.zeros_like(ct)
        self.L.ref_hg_eval(g, _p(ct), len(ct), _p(out))
        return out

    def hg_sample(self, g, iv, u1, u2):
        iv = np.ascontiguousarray(iv, np.float32).reshape(-1, 3)
        u1 = np.ascontiguousarray(u1, np.float32)
        u2 = np.ascontiguousarray(u2, np.float32)
        out = np.zeros_like(iv)
        self.L.ref_hg_sample(g, _p(iv), _p(u1), _p(u2), len(iv), _p(out))
        return out

    def atan2(self, y, x):
        y = np.ascontiguousarray(y, np.float32)
        x = np.ascontiguousarray(x, np.float32)
        out = np.zeros_like(y)
        self.L.ref_atan2(_p(y), _p(x), len(y), _p(out))
        return out

    def env_eval(self, env_map, rd):
        em = np.ascontiguousarray(env_map, np.float32)
        rd = np.ascontiguousarray(rd, np.float32).reshape(-1, 3)
        out = np.zeros_like(rd)
        self.L.ref_env_eval(em.shape[1], em.shape[0], _p(em), _p(rd), len(rd), _p(out))
        return out

    def set_threads(self, n: int):
        self.L.ref_set_threads(int(n))

    def scene(self, nodes: np.ndarray, bricks: np.ndarray, sdf: np.ndarray = None):
        nodes = np.ascontiguousarray(nodes)
        bricks = np.ascontiguousarray(bricks, np.float32)
        if sdf is None:
            return _RefScene(self, self.L.ref_scene_create(_p(nodes), len(nodes), _p(bricks), len(bricks), 8))
        sdf = np.ascontiguousarray(sdf, np.float32).reshape(-1, 512)
        return _RefScene(self, self.L.ref_scene_create_sdf(_p(nodes), len(nodes), _p(bricks), len(bricks), _p(sdf),
                                                           len(sdf), 8))

    def mie_tables(self):
        n = self.L.ref_mie_table_size()
        pdf = np.zeros((n, 3), np.float32)
        cdf = np.zeros((n, 3), np.float32)
        self.L.ref_mie_tables(_p(pdf), _p(cdf))
        return pdf, cdf

    def sky_state(self, turbidity, albedo, elevation):
        cfg = np.zeros((3, 9), np.float64)
        rad = np.zeros(3, np.float64)
        self.L.ref_sky_state(turbidity, albedo, elevation, _p(cfg), _p(rad))
        return cfg, rad

    def solar_elevation(self, sun_dir):
        s = np.ascontiguousarray(sun_dir, np.float32)
        return float(self.L.ref_solar_elevation(_p(s)))

    def sample_voxel_space(self, p, brick, ce):
        p = np.ascontiguousarray(p, np.float32)
        brick = np.ascontiguousarray(brick, np.float32)
        ce = np.ascontiguousarray(ce, np.float32)
        return float(self.L.ref_sample_voxel_space(_p(p), _p(brick), _p(ce), 8))

    def mie_eval(self, ct):
        ct = np.ascontiguousarray(ct, np.float32)
        s = np.zeros(len(ct), np.float32)
        rgb = np.zeros((len(ct), 3), np.float32)
        self.L.ref_mie_eval(_p(ct), len(ct), _p(s), _p(rgb))
        return s, rgb

    def mie_sample(self, iv, u1, u2):
        iv = np.ascontiguousarray(iv, np.float32)
        u1 = np.ascontiguousarray(u1, np.float32)
        u2 = np.ascontiguousarray(u2, np.float32)
        out = np.zeros((len(u1), 3), np.float32)
        self.L.ref_mie_sample(_p(iv), _p(u1), _p(u2), len(u1), _p(out))
        return out

    def sun_ops(self, sun_dir, color, angle, v, u1, u2):
        d = np.ascontiguousarray(sun_dir, np.float32)
        c = np.ascontiguousarray(color, np.float32)
        v = np.ascontiguousarray(v, np.float32)
        u1 = np.ascontiguousarray(u1, np.float32)
        u2 = np.ascontiguousarray(u2, np.float32)
        n = len(u1)
        ev = np.zeros((n, 3), np.float32)
        pdf = np.zeros(n, np.float32)
        smp = np.zeros((n, 3), np.float32)
        self.L.ref_sun_ops(_p(d), _p(c), angle, _p(v), _p(u1), _p(u2), n, _p(ev), _p(pdf), _p(smp))
        return ev, pdf, smp


class _RefScene:
    def __init__(self, ref: Reference, handle):
        self.ref = ref
        self.h = handle

    def __del__(self):
        if getattr(self, "h", None):
            self.ref.L.ref_scene_destroy(self.h)
            self.h = None

    def leaf_sequence(self, ro, rd, full=False, maxn=4096):
        ro = np.ascontiguousarray(ro, np.float32)
        rd = np.ascontiguousarray(rd, np.float32)
        n_ = np.zeros(maxn, np.uint32)
        a = np.zeros(maxn, np.float32)
        b = np.zeros(maxn, np.float32)
        k = self.ref.L.ref_leaf_sequence(self.h, 1 if full else 0, _p(ro), _p(rd), maxn, _p(n_), _p(a), _p(b))
        return n_[:k], a[:k], b[:k]

    def render(self, cfg: dict, x0, y0, tw, th, spp):
        """RenderKernel::Render over one tile; returns (sun, sky) float4 tiles (sums over spp)."""
        viewi = np.ascontiguousarray(cfg["viewi"], np.float32)
        proji = np.ascontiguousarray(cfg["proji"], np.float32)
        sd = np.ascontiguousarray(cfg["sun_dir"], np.float32)
        sc = np.ascontiguousarray(cfg["sun_color"], np.float32)
        sun = np.zeros((th, tw, 4), np.float32)
        sky = np.zeros((th, tw, 4), np.float32)
        depth = None if cfg.get("depth") is None else np.ascontiguousarray(cfg["depth"], np.float32).reshape(-1)
        rc = self.ref.L.ref_render(self.h, _p(viewi), _p(proji), _p(sd), _p(sc), float(cfg["sun_angle"]),
                                   float(cfg["turbidity"]), float(cfg["ground_albedo"]), int(cfg["scattevs"]),
                                   float(cfg["sigma_s"]), float(cfg["sigma_a"]), int(cfg["w"]), int(cfg["h"]),
                                   x0, y0, tw, th, spp, _p(sun), _p(sky), None if depth is None else _p(depth),
                                   1 if cfg.get("depthcomp") else 0)
        if rc != 0:
            raise RuntimeError("ref_render failed")
        return sun, sky

    def render_ex(self, cfg: dict, x0, y0, tw, th, spp):
        """render() with the phase function (cfg phase_mode 2 = HG, hg_g) and the
        environment map (cfg env_mode 2, env_map (h, w, 4)) of the configuration."""
        viewi = np.ascontiguousarray(cfg["viewi"], np.float32)
        proji = np.ascontiguousarray(cfg["proji"], np.float32)
        sd = np.ascontiguousarray(cfg["sun_dir"], np.float32)
        sc = np.ascontiguousarray(cfg["sun_color"], np.float32)
        sun = np.zeros((th, tw, 4), np.float32)
        sky = np.zeros((th, tw, 4), np.float32)
        depth = None if cfg.get("depth") is None else np.ascontiguousarray(cfg["depth"], np.float32).reshape(-1)
        em = None
        if cfg.get("env_mode", 0) == 2:
            em = np.ascontiguousarray(cfg["env_map"], np.float32)
        rc = self.ref.L.ref_render_ex(self.h, _p(viewi), _p(proji), _p(sd), _p(sc), float(cfg["sun_angle"]),
                                      float(cfg["turbidity"]), float(cfg["ground_albedo"]), int(cfg["scattevs"]),
                                      float(cfg["sigma_s"]), float(cfg["sigma_a"]), int(cfg["w"]), int(cfg["h"]),
                                      x0, y0, tw, th, spp, _p(sun), _p(sky), None if depth is None else _p(depth),
                                      1 if cfg.get("depthcomp") else 0, 2 if cfg.get("phase_mode", 0) == 2 else 0,
                                      float(cfg.get("hg_g", 0.0)), 0 if em is None else em.shape[1],
                                      0 if em is None else em.shape[0], None if em is None else _p(em))
        if rc != 0:
            raise RuntimeError("ref_render_ex failed")
        return sun, sky

    def shadow(self, cfg: dict, x0, y0, tw, th, spp):
        """RenderKernel::Shadow over one tile; returns the phb[0] float4 tile (sums over spp)."""
        viewi = np.ascontiguousarray(cfg["viewi"], np.float32)
        proji = np.ascontiguousarray(cfg["proji"], np.float32)
        sd = np.ascontiguousarray(cfg["sun_dir"], np.float32)
        sc = np.ascontiguousarray(cfg["sun_color"], np.float32)
        out = np.zeros((th, tw, 4), np.float32)
        depth = None if cfg.get("depth") is None else np.ascontiguousarray(cfg["depth"], np.float32).reshape(-1)
        rc = self.ref.L.ref_shadow(self.h, _p(viewi), _p(proji), _p(sd), _p(sc), float(cfg["sun_angle"]),
                                   int(cfg["scattevs"]), float(cfg["sigma_s"]), float(cfg["sigma_a"]), int(cfg["w"]),
                                   int(cfg["h"]), x0, y0, tw, th, spp, None if depth is None else _p(depth), _p(out))
        if rc != 0:
            raise RuntimeError("ref_shadow failed")
        return out
