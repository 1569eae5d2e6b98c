"""Hosek-Wilkie sky state for the renderer.

The kernel consumes the cooked RGB state exactly as the reference's
RenderKernel reads ArHosekSkyModelState (src/kernel.cpp:343-358): nine
coefficients and one radiance scale per channel.  The cook itself
(src/ArHosekSkyModel.cpp:147-339) runs in the native library
(dr_sky_cook) on the Hosek-Wilkie RGB dataset, which the caller supplies:
`load_dataset` reads it from the C header that ships with the model's
reference implementation (datasetRGB1..3, datasetRGBRad1..3).
"""
from __future__ import annotations

import ctypes as C
import re
from dataclasses import dataclass

import numpy as np

from . import _native as N


@dataclass
class SkyState:
    configs: np.ndarray      # (3, 9) float64
    radiances: np.ndarray    # (3,) float64

    def as_dict(self):
        return {"configs": self.configs.tolist(), "radiances": self.radiances.tolist()}

    @staticmethod
    def from_dict(d) -> "SkyState":
        return SkyState(np.asarray(d["configs"], np.float64).reshape(3, 9), np.asarray(d["radiances"], np.float64))


def solar_elevation(sun_dir) -> float:
    """pi/2 - acos(sun.z) in binary32, as RenderKernel::Initialize does (src/kernel.cpp:522-524)."""
    z = np.float32(sun_dir[2])
    th = np.float32(np.arccos(z))
    return float(np.float32(1.570796327) - th)


def load_dataset(header_path: str):
    """Parses datasetRGB1..3 (1080 doubles each) and datasetRGBRad1..3 (120) from the model's C header."""
    text = open(header_path, "r", encoding="utf-8", errors="replace").read()
    num = re.compile(r"[-+]?\d+\.?\d*(?:[eE][-+]?\d+)?")

    def grab(name: str, n: int) -> np.ndarray:
        m = re.search(r"double\s+" + name + r"\s*\[\s*\]\s*=\s*\{(.*?)\}\s*;", text, re.S)
        if not m:
            raise ValueError(f"{header_path}: no table {name}")
        body = re.sub(r"//[^\n]*", "", m.group(1))
        vals = np.array([float(v) for v in num.findall(body)], np.float64)
        if vals.size != n:
            raise ValueError(f"{header_path}: table {name} has {vals.size} values, expected {n}")
        return vals

    rgb = [grab(f"datasetRGB{c}", 1080) for c in (1, 2, 3)]
    rad = [grab(f"datasetRGBRad{c}", 120) for c in (1, 2, 3)]
    return rgb, rad


def cook(dataset, turbidity: float, albedo: float, elevation: float) -> SkyState:
    rgb, rad = dataset
    rgb = [np.ascontiguousarray(a, np.float64) for a in rgb]
    rad = [np.ascontiguousarray(a, np.float64) for a in rad]
    p_rgb = (C.c_void_p * 3)(*[a.ctypes.data for a in rgb])
    p_rad = (C.c_void_p * 3)(*[a.ctypes.data for a in rad])
    cfg = np.zeros((3, 9), np.float64)
    radi = np.zeros(3, np.float64)
    N.check(N.lib().dr_sky_cook(p_rgb, p_rad, float(turbidity), float(albedo), float(elevation),
                                cfg.ctypes.data, radi.ctypes.data))
    return SkyState(cfg, radi)
