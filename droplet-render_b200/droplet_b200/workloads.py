"""Seeded synthetic density fields for the benchmark and tests.

Recipe (one "puff"): density(p) = max(0, 1 - |p - c| / R) * fBm(p), where fBm
is 4-octave gradient noise (base frequency 4, lacunarity 2, gain 0.5, amp 1)
and the total is clamped to [0, 1].  The noise is Perlin's improved gradient
noise (Perlin 2002: quintic fade, 12 cube-edge gradients selected by the low
hash bits); its "seed" selects the permutation table, drawn with
numpy.random.default_rng(seed).permutation(256).  Voxel (i, j, k) of an n^3
grid on the unit cube sits at world (i, j, k) / n, as the reference's
uniform-scale transform places it.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def perm_table(seed: int) -> np.ndarray:
    p = np.random.default_rng(seed).permutation(256).astype(np.int64)
    return np.concatenate([p, p])


def _fade(t):
    return t * t * t * (t * (t * 6.0 - 15.0) + 10.0)


def _grad(h, x, y, z):
    h = h & 15
    u = np.where(h < 8, x, y)
    v = np.where(h < 4, y, np.where((h == 12) | (h == 14), x, z))
    return np.where(h & 1, -u, u) + np.where(h & 2, -v, v)


def perlin(x, y, z, perm):
    """Improved gradient noise at float64 points (arrays of one shape)."""
    xf, yf, zf = np.floor(x), np.floor(y), np.floor(z)
    X = xf.astype(np.int64) & 255
    Y = yf.astype(np.int64) & 255
    Z = zf.astype(np.int64) & 255
    x, y, z = x - xf, y - yf, z - zf
    u, v, w = _fade(x), _fade(y), _fade(z)
    A = perm[X] + Y
    AA = perm[A] + Z
    AB = perm[A + 1] + Z
    B = perm[X + 1] + Y
    BA = perm[B] + Z
    BB = perm[B + 1] + Z

    def lerp(t, a, b):
        return a + t * (b - a)

    return lerp(
        w,
        lerp(v, lerp(u, _grad(perm[AA], x, y, z), _grad(perm[BA], x - 1, y, z)),
             lerp(u, _grad(perm[AB], x, y - 1, z), _grad(perm[BB], x - 1, y - 1, z))),
        lerp(v, lerp(u, _grad(perm[AA + 1], x, y, z - 1), _grad(perm[BA + 1], x - 1, y, z - 1)),
             lerp(u, _grad(perm[AB + 1], x, y - 1, z - 1), _grad(perm[BB + 1], x - 1, y - 1, z - 1))),
    )


def fbm(x, y, z, seed: int, octaves: int = 4, freq: float = 4.0, lacunarity: float = 2.0, gain: float = 0.5):
    perm = perm_table(seed)
    s = np.zeros_like(x)
    amp = 1.0
    for _ in range(octaves):
        s += amp * perlin(x * freq, y * freq, z * freq, perm)
        freq *= lacunarity
        amp *= gain
    return s


@dataclass
class Puff:
    center: tuple
    radius: float
    seed: int


@dataclass
class FieldRecipe:
    n: int                       # grid edge (voxels)
    puffs: list = field(default_factory=list)
    extent: tuple = (1.0, 1.0, 1.0)  # fraction of the unit cube covered per axis (slabs)

    @property
    def voxel_size(self) -> float:
        return 1.0 / self.n


def config0_recipe(n: int = 64, seed: int = 1) -> FieldRecipe:
    """Single puff at the cube centre, radius 0.4."""
    return FieldRecipe(n, [Puff((0.5, 0.5, 0.5), 0.4, seed)])


def slab_recipe(n: int = 2048, seed: int = 2044, count: int = 24) -> FieldRecipe:
    """The large sparse scene: `count` config-0-style puffs (seeds 20-43, radii
    uniform in [0.02, 0.12], default_rng(seed) draws) inside a slab 1 x 1 wide and
    0.3 thick along z (the up axis), centred at z = 0.5; each sphere lies inside
    the slab.  On a 2048^3 grid about 2% of the voxels are non-empty."""
    rng = np.random.default_rng(seed)
    puffs = []
    for k in range(count):
        r = float(rng.uniform(0.02, 0.12))
        c = (float(rng.uniform(r, 1.0 - r)), float(rng.uniform(r, 1.0 - r)), float(rng.uniform(0.35 + r, 0.65 - r)))
        puffs.append(Puff(c, r, 20 + k))
    return FieldRecipe(n, puffs, extent=(1.0, 1.0, 0.3))


def cumulus_recipe(n: int = 512) -> FieldRecipe:
    """The config-0 puff plus three offset, scaled copies (radii 0.15-0.3, seeds 2-4)."""
    return FieldRecipe(
        n,
        [
            Puff((0.5, 0.5, 0.5), 0.4, 1),
            Puff((0.3, 0.42, 0.58), 0.25, 2),
            Puff((0.72, 0.56, 0.54), 0.22, 3),
            Puff((0.52, 0.38, 0.74), 0.15, 4),
        ],
    )


# Scene setup shared by the configurations: camera 2.5 units from the cube
# centre with a 40 degree vertical field of view, sun at 30 degrees elevation
# (white, intensity 1 and cone half-angle 0.010 rad, the reference UI
# defaults, addon/panel.py:360-362), Hosek sky with turbidity 3 and ground
# albedo 0.3.
CENTER = (0.5, 0.5, 0.5)
CAMERA = {"distance": 2.5, "azimuth": -90.0, "elevation": 10.0, "fov": 40.0}
SUN = {"elevation": 30.0, "azimuth": 30.0, "color": (1.0, 1.0, 1.0), "angle": 0.010}
SKY = {"turbidity": 3.0, "albedo": 0.3}
MEDIA = {
    "c0": {"sigma_t": 20.0, "albedo": 0.99, "scattevs": 8},
    "c1": {"sigma_t": 60.0, "albedo": 0.999, "scattevs": 64},
    "c4": {"sigma_t": 100.0, "albedo": 0.99, "scattevs": 128},
}
# The batched workload's fields take their own sigma_t; albedo as config 0 and
# the reference UI's default of 500 scattering events.
C2_ALBEDO, C2_SCATTEVS = 0.99, 500


def medium(name: str):
    """(sigma_s, sigma_a, scattevs) in binary32 for a named configuration."""
    m = MEDIA[name]
    return medium_of(m["sigma_t"], m["albedo"], m["scattevs"])


def medium_of(sigma_t: float, albedo: float, scattevs: int):
    st = np.float32(sigma_t)
    ss = np.float32(sigma_t * albedo)
    return float(ss), float(np.float32(st - ss)), int(scattevs)


def c2_batch(seed: int = 2026):
    """The batched workload (8 fields x 8 views), drawn with default_rng(seed).

    Fields: the config-0 puff recipe at seeds 10-17, grid edge from
    {64, 128, 256, 512}, sigma_t uniform in [10, 80].  Views: 8 per field at
    uniform random azimuths (camera 2.5 units from the centre, 10 degrees up,
    40 degree field of view), square images with an even side uniform in
    [128, 1024], spp from {16, 64, 256}, and the sun (azimuth 30) at a whole
    degree of elevation uniform in [5, 80] (the sky states are cooked per
    degree).  Returns (fields, views) as lists of dicts."""
    rng = np.random.default_rng(seed)
    fields = [{"seed": 10 + i, "n": int(rng.choice([64, 128, 256, 512])),
               "sigma_t": float(rng.uniform(10.0, 80.0))} for i in range(8)]
    views = []
    for f in range(8):
        for _ in range(8):
            views.append({"field": f, "azimuth": float(rng.uniform(0.0, 360.0)),
                          "side": 2 * int(rng.integers(64, 513)), "spp": int(rng.choice([16, 64, 256])),
                          "sun_elevation": int(rng.integers(5, 81))})
    return fields, views


def eval_blocks_numpy(recipe: FieldRecipe, block_origins: np.ndarray, chunk: int = 2048) -> np.ndarray:
    """Density of 8^3 blocks (x fastest) at the given block origins; float32."""
    o_all = np.asarray(block_origins, np.int64).reshape(-1, 3)
    if len(o_all) > chunk:
        return np.concatenate([eval_blocks_numpy(recipe, o_all[c:c + chunk], chunk)
                               for c in range(0, len(o_all), chunk)])
    s = recipe.voxel_size
    o = o_all
    k, j, i = np.meshgrid(np.arange(8), np.arange(8), np.arange(8), indexing="ij")
    ii = (o[:, 0, None] + i.reshape(1, -1)).astype(np.float64)
    jj = (o[:, 1, None] + j.reshape(1, -1)).astype(np.float64)
    kk = (o[:, 2, None] + k.reshape(1, -1)).astype(np.float64)
    x, y, z = ii * s, jj * s, kk * s
    total = np.zeros_like(x)
    for p in recipe.puffs:
        r = np.sqrt((x - p.center[0]) ** 2 + (y - p.center[1]) ** 2 + (z - p.center[2]) ** 2)
        env = np.maximum(0.0, 1.0 - r / p.radius)
        m = env > 0
        if m.any():
            total[m] += env[m] * fbm(x[m], y[m], z[m], p.seed)
    return np.clip(total, 0.0, 1.0).astype(np.float32)


def _grad_t(h, x, y, z):
    import torch

    h = h & 15
    u = torch.where(h < 8, x, y)
    v = torch.where(h < 4, y, torch.where((h == 12) | (h == 14), x, z))
    return torch.where((h & 1) != 0, -u, u) + torch.where((h & 2) != 0, -v, v)


def _fade_t(t):
    return t * t * t * (t * (t * 6.0 - 15.0) + 10.0)


def _lerp_t(t, a, b):
    return a + t * (b - a)


def _perlin_t(x, y, z, perm):
    """perlin() on torch float64 tensors (same operations)."""
    import torch

    xf, yf, zf = torch.floor(x), torch.floor(y), torch.floor(z)
    X = xf.long() & 255
    Y = yf.long() & 255
    Z = zf.long() & 255
    x, y, z = x - xf, y - yf, z - zf
    u, v, w = _fade_t(x), _fade_t(y), _fade_t(z)
    A = perm[X] + Y
    AA = perm[A] + Z
    AB = perm[A + 1] + Z
    B = perm[X + 1] + Y
    BA = perm[B] + Z
    BB = perm[B + 1] + Z
    return _lerp_t(w,
                   _lerp_t(v, _lerp_t(u, _grad_t(perm[AA], x, y, z), _grad_t(perm[BA], x - 1, y, z)),
                           _lerp_t(u, _grad_t(perm[AB], x, y - 1, z), _grad_t(perm[BB], x - 1, y - 1, z))),
                   _lerp_t(v, _lerp_t(u, _grad_t(perm[AA + 1], x, y, z - 1), _grad_t(perm[BA + 1], x - 1, y, z - 1)),
                           _lerp_t(u, _grad_t(perm[AB + 1], x, y - 1, z - 1),
                                   _grad_t(perm[BB + 1], x - 1, y - 1, z - 1))))


def _puff_term_t(p, x, y, z, perm):
    """(mask, env * fBm) of one puff at the voxels (x, y, z): float64 tensors."""
    import torch

    r = torch.sqrt((x - p.center[0]) ** 2 + (y - p.center[1]) ** 2 + (z - p.center[2]) ** 2)
    env = torch.clamp(1.0 - r / p.radius, min=0.0)
    m = env > 0
    xs, ys, zs = x[m], y[m], z[m]
    acc = torch.zeros_like(xs)
    amp, freq = 1.0, 4.0
    for _ in range(4):
        acc += amp * _perlin_t(xs * freq, ys * freq, zs * freq, perm)
        freq *= 2.0
        amp *= 0.5
    return m, env[m] * acc


def eval_blocks_torch(recipe: FieldRecipe, block_origins: np.ndarray, device="cuda", chunk: int = 8192) -> np.ndarray:
    """eval_blocks_numpy with torch float64 tensors (same operations in the same
    order, so the same values), for building large fields quickly on a GPU."""
    import torch

    s = recipe.voxel_size
    org_all = torch.as_tensor(np.asarray(block_origins, np.int64).reshape(-1, 3), device=device)
    k, j, i = torch.meshgrid(torch.arange(8, device=device), torch.arange(8, device=device),
                             torch.arange(8, device=device), indexing="ij")
    i, j, k = i.reshape(1, -1), j.reshape(1, -1), k.reshape(1, -1)
    perms = {p.seed: torch.as_tensor(perm_table(p.seed), device=device) for p in recipe.puffs}
    out = []
    for c0 in range(0, org_all.shape[0], chunk):
        o = org_all[c0:c0 + chunk]
        x = (o[:, 0:1] + i).double() * s
        y = (o[:, 1:2] + j).double() * s
        z = (o[:, 2:3] + k).double() * s
        total = torch.zeros_like(x)
        for p in recipe.puffs:
            m, term = _puff_term_t(p, x, y, z, perms[p.seed])
            if bool(m.any()):
                total[m] += term
        out.append(torch.clamp(total, 0.0, 1.0).float().cpu().numpy())
    return np.concatenate(out) if out else np.zeros((0, 512), np.float32)


def puff_blocks(recipe: FieldRecipe, p) -> np.ndarray:
    """Origins of the 8^3 blocks of the grid that intersect one puff's sphere."""
    n, s = recipe.n, recipe.voxel_size
    nb = (n + 7) // 8
    c = np.asarray(p.center, np.float64)
    lo = np.clip(np.floor((c - p.radius) / s / 8).astype(np.int64), 0, nb - 1)
    hi = np.clip(np.floor((c + p.radius) / s / 8).astype(np.int64), 0, nb - 1)
    g = [np.arange(lo[a], hi[a] + 1) * 8 for a in range(3)]
    bx, by, bz = np.meshgrid(g[0], g[1], g[2], indexing="ij")
    org = np.stack([bx.ravel(), by.ravel(), bz.ravel()], -1)
    blo = org * s
    bhi = (org + 7) * s
    d = np.maximum(0.0, np.maximum(blo - c, c - bhi))
    return org[np.sqrt((d ** 2).sum(-1)) < p.radius]


def sparse_field_puffwise(recipe: FieldRecipe, device="cuda", chunk: int = 16384):
    """sparse_field for many small puffs in a large grid: each puff is evaluated
    only on its own blocks and the terms are summed per voxel in puff order (the
    values of eval_blocks_numpy).  Returns (block_origins, block_values) of the
    non-empty blocks, sorted by block origin."""
    import torch

    per = [puff_blocks(recipe, p) for p in recipe.puffs]
    allb = np.concatenate(per) if per else np.zeros((0, 3), np.int64)
    uniq, inv = np.unique(allb, axis=0, return_inverse=True)
    inv = inv.reshape(-1)
    s = recipe.voxel_size
    total = torch.zeros((len(uniq), 512), dtype=torch.float64, device=device)
    k, j, i = torch.meshgrid(torch.arange(8, device=device), torch.arange(8, device=device),
                             torch.arange(8, device=device), indexing="ij")
    i, j, k = i.reshape(1, -1), j.reshape(1, -1), k.reshape(1, -1)
    off = 0
    for p, blocks in zip(recipe.puffs, per):
        perm = torch.as_tensor(perm_table(p.seed), device=device)
        rows_all = torch.as_tensor(inv[off:off + len(blocks)], device=device)
        off += len(blocks)
        ob = torch.as_tensor(blocks, device=device)
        for c0 in range(0, len(blocks), chunk):
            o = ob[c0:c0 + chunk]
            rows = rows_all[c0:c0 + chunk]
            x = (o[:, 0:1] + i).double() * s
            y = (o[:, 1:2] + j).double() * s
            z = (o[:, 2:3] + k).double() * s
            m, term = _puff_term_t(p, x, y, z, perm)
            full = torch.zeros_like(x)
            full[m] = term
            total.index_add_(0, rows, full)
    vals = torch.clamp(total, 0.0, 1.0).float()
    nz = (vals != 0).any(1).cpu().numpy()
    return np.ascontiguousarray(uniq[nz].astype(np.int32)), np.ascontiguousarray(vals.cpu().numpy()[nz])


def sparse_field_fast(recipe: FieldRecipe):
    """sparse_field using a CUDA device when torch sees one, numpy otherwise."""
    try:
        import torch

        use_cuda = torch.cuda.is_available()
    except Exception:
        use_cuda = False
    if not use_cuda:
        return sparse_field(recipe)
    org = candidate_blocks(recipe)
    vals = eval_blocks_torch(recipe, org)
    nz = (vals != 0).any(1)
    return np.ascontiguousarray(org[nz]), np.ascontiguousarray(vals[nz])


def candidate_blocks(recipe: FieldRecipe) -> np.ndarray:
    """Origins of the 8^3 blocks that intersect any puff's bounding sphere."""
    n, s = recipe.n, recipe.voxel_size
    nb = (n + 7) // 8
    g = np.arange(nb) * 8
    bx, by, bz = np.meshgrid(g, g, g, indexing="ij")
    org = np.stack([bx.ravel(), by.ravel(), bz.ravel()], -1)
    keep = np.zeros(len(org), bool)
    lo = org * s
    hi = (org + 7) * s
    for p in recipe.puffs:
        c = np.asarray(p.center)
        d = np.maximum(0.0, np.maximum(lo - c, c - hi))
        keep |= np.sqrt((d ** 2).sum(-1)) < p.radius
    return org[keep].astype(np.int32)


def sparse_field(recipe: FieldRecipe):
    """(block_origins int32 (B,3), block_values float32 (B,512)) of the non-empty blocks."""
    org = candidate_blocks(recipe)
    vals = eval_blocks_numpy(recipe, org) if len(org) else np.zeros((0, 512), np.float32)
    nz = (vals != 0).any(1)
    return np.ascontiguousarray(org[nz]), np.ascontiguousarray(vals[nz])


def dense_to_blocks(grid: np.ndarray):
    """Dense (nz, ny, nx) -> ... ; grid indexed [x, y, z] with shape multiple of 8."""
    g = np.asarray(grid, np.float32)
    nx, ny, nz = g.shape
    px, py, pz = (-nx) % 8, (-ny) % 8, (-nz) % 8
    if px or py or pz:
        g = np.pad(g, ((0, px), (0, py), (0, pz)))
    bx, by, bz = g.shape[0] // 8, g.shape[1] // 8, g.shape[2] // 8
    b = g.reshape(bx, 8, by, 8, bz, 8).transpose(0, 2, 4, 5, 3, 1)  # (bx,by,bz, z, y, x)
    b = b.reshape(bx * by * bz, 512)
    ox, oy, oz = np.meshgrid(np.arange(bx) * 8, np.arange(by) * 8, np.arange(bz) * 8, indexing="ij")
    org = np.stack([ox.ravel(), oy.ravel(), oz.ravel()], -1).astype(np.int32)
    nzm = (b != 0).any(1)
    return np.ascontiguousarray(org[nzm]), np.ascontiguousarray(b[nzm])
