"""Camera matrices in the reference's conventions.

DRE_BeginRender (src/main.cpp:71-115) builds
    view = XMMatrixLookToRH(p, d, u),  u = (0, 0, -1), d = rotate(u, q)
    proj = XMMatrixPerspectiveRH(frx, fry, clip_start, clip_end)
and hands their inverses (row-vector convention, rows r[0..3]) to the kernel.
The ray for pixel (px, py) is normalize(((posh P^-1).xyz, 0) V^-1) from the
origin V^-1.r[3] (src/kernel.cpp:461-470).  This module builds the same
matrices for a camera placed at `eye` looking at `target` with a vertical
field of view, so a view frame of 2 n tan(fov/2) (x aspect) at the near plane.
"""
from __future__ import annotations

import numpy as np

UP = np.array([0.0, 0.0, -1.0])


def look_to_rh(eye, d, up=UP) -> np.ndarray:
    """XMMatrixLookToRH (SMMathPort.inl:494-512) in float64, row-vector convention."""
    eye = np.asarray(eye, np.float64)
    r2 = -np.asarray(d, np.float64)
    r2 = r2 / np.linalg.norm(r2)
    r0 = np.cross(up, r2)
    r0 = r0 / np.linalg.norm(r0)
    r1 = np.cross(r2, r0)
    m = np.zeros((4, 4))
    m[0, :3], m[0, 3] = r0, np.dot(r0, -eye)
    m[1, :3], m[1, 3] = r1, np.dot(r1, -eye)
    m[2, :3], m[2, 3] = r2, np.dot(r2, -eye)
    m[3] = [0, 0, 0, 1]
    return m.T.copy()


def perspective_rh(view_w: float, view_h: float, near: float, far: float) -> np.ndarray:
    """XMMatrixPerspectiveRH (SMMathPort.inl:374-413)."""
    frange = far / (near - far)
    m = np.zeros((4, 4))
    m[0, 0] = 2.0 * near / view_w
    m[1, 1] = 2.0 * near / view_h
    m[2, 2] = frange
    m[2, 3] = -1.0
    m[3, 2] = frange * near
    return m


def camera_matrices(eye, target, fov_y_deg: float, w: int, h: int, near: float = 0.1, far: float = 100.0):
    """Inverse view and inverse projection (16 float32 each, rows r[0..3])."""
    eye = np.asarray(eye, np.float64)
    d = np.asarray(target, np.float64) - eye
    view = look_to_rh(eye, d)
    t = np.tan(np.radians(fov_y_deg) * 0.5)
    proj = perspective_rh(2.0 * near * t * (w / h), 2.0 * near * t, near, far)
    viewi = np.linalg.inv(view).astype(np.float32)
    proji = np.linalg.inv(proj).astype(np.float32)
    return viewi.reshape(16), proji.reshape(16)


def orbit_eye(center, distance: float, azimuth_deg: float, elevation_deg: float = 0.0) -> np.ndarray:
    """Camera position on a sphere around `center` (z up)."""
    az, el = np.radians(azimuth_deg), np.radians(elevation_deg)
    c = np.asarray(center, np.float64)
    return c + distance * np.array([np.cos(el) * np.cos(az), np.cos(el) * np.sin(az), np.sin(el)])


def sun_direction(elevation_deg: float, azimuth_deg: float = 0.0) -> np.ndarray:
    """Unit vector towards the sun (z up), float32."""
    el, az = np.radians(elevation_deg), np.radians(azimuth_deg)
    v = np.array([np.cos(el) * np.cos(az), np.cos(el) * np.sin(az), np.sin(el)])
    return (v / np.linalg.norm(v)).astype(np.float32)


def camera_rays(viewi, proji, w: int, h: int, px, py):
    """Float32 restatement of the kernel's ray generation (for host-side checks)."""
    V = np.asarray(viewi, np.float32).reshape(4, 4)
    Q = np.asarray(proji, np.float32).reshape(4, 4)
    px = np.asarray(px, np.float32)
    py = np.asarray(py, np.float32)
    one = np.float32(1)
    hx = np.float32(0) - ((np.float32(2) * (px + np.float32(0.5))) / np.float32(w) - one)
    hy = np.float32(0) - ((np.float32(2) * (py + np.float32(0.5))) / np.float32(h) - one)
    rv = [((hx * Q[0, k] + hy * Q[1, k]) + np.float32(0) * Q[2, k]) + one * Q[3, k] for k in range(3)]
    d = [((rv[0] * V[0, k] + rv[1] * V[1, k]) + rv[2] * V[2, k]) + np.float32(0) * V[3, k] for k in range(3)]
    ln = np.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
    rd = np.stack([d[k] / ln for k in range(3)], -1)
    ro = np.broadcast_to(V[3, :3], rd.shape).copy()
    inside = (hx > -1) & (hx < 1) & (hy > -1) & (hy < 1)
    return ro, rd, inside
