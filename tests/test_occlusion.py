"""Holdout-mesh occlusion (SceneOcclusion, src/SceneOcclusion.cpp:19-91) without a
GPU: the host BVH the library builds (every selected triangle exactly once,
inside the boxes on its way down, the holdout selection of both modes), the
CPU restatement's binary32 triangle test against an FP64 test away from
edges, and the restatement's render semantics: occluders act only in the
USE_EMBREE build, where they zero the light that escaping segments gather,
and that build's depth mask zeroes the alpha of a camera ray cut at its depth.

Embree itself is not in the reference tree and cannot run here, so the
occlusion answer is pinned to FP64 geometry, not to Embree's arithmetic."""
import numpy as np

from conftest import c0_cfg, depth_texture, golden_octree, occluder_surfaces
from droplet_b200.renderer import OCCLUDE_ALL_SURFACES, OCCLUDE_HOLDOUT_ONLY, build_occluder_bvh


def _children(node):
    w = node[12:16].view(np.uint32)
    return [(node[0:6], int(w[0]), int(w[2])), (node[6:12], int(w[1]), int(w[3]))]


def _inside(box, pts):
    return bool(((pts >= box[:3]) & (pts <= box[3:])).all())


def test_bvh_holds_every_selected_triangle_once_inside_its_boxes():
    surfaces = occluder_surfaces()
    nodes, tris, src = build_occluder_bvh(surfaces, OCCLUDE_ALL_SURFACES)
    total = sum(len(ix) for _, ix, _ in surfaces)
    assert len(tris) == total and sorted(src.tolist()) == list(range(total))
    # triangle data: (v0, v1 - v0, v2 - v0) of its source triangle, in binary32
    flat = [(v, t) for v, ix, _ in surfaces for t in ix]
    for j in range(0, total, 7):
        v, t = flat[src[j]]
        v0, v1, v2 = (np.asarray(v[t[k]], np.float32) for k in range(3))
        assert np.array_equal(tris[j, 0:3], v0)
        assert np.array_equal(tris[j, 4:7], v1 - v0) and np.array_equal(tris[j, 8:11], v2 - v0)
    seen = np.zeros(total, int)
    # walk: every triangle inside every box on its way down; depth within the cap
    stack = [(0, 0)]
    visited = 0
    while stack:
        n, depth = stack.pop()
        visited += 1
        assert depth < 48
        for box, ref, count in _children(nodes[n]):
            if ref == 0xFFFFFFFF:
                continue
            if count:
                for j in range(ref, ref + count):
                    seen[j] += 1
                    corners = np.stack([tris[j, 0:3], tris[j, 0:3] + tris[j, 4:7], tris[j, 0:3] + tris[j, 8:11]])
                    assert _inside(box, corners)
            else:
                # the child's own child boxes (same padding) lie inside this box
                for cbox, cref, _ in _children(nodes[ref]):
                    if cref != 0xFFFFFFFF:
                        assert (cbox[:3] >= box[:3]).all() and (cbox[3:] <= box[3:]).all()
                stack.append((ref, depth + 1))
    assert visited == len(nodes)
    assert (seen == 1).all()


def test_holdout_only_mode_selects_flagged_surfaces():
    surfaces = occluder_surfaces()
    _, tris, src = build_occluder_bvh(surfaces, OCCLUDE_HOLDOUT_ONLY)
    flagged = sum(len(ix) for _, ix, f in surfaces if f & 2)
    assert len(tris) == flagged < sum(len(ix) for _, ix, _ in surfaces)
    nodes, tris, src = build_occluder_bvh([], OCCLUDE_ALL_SURFACES)
    assert len(nodes) == 0 and len(tris) == 0


def _rays(n, seed):
    rng = np.random.default_rng(seed)
    ro = rng.uniform([-0.5, -0.5, 0.1], [2.0, 2.0, 1.5], (n, 3))
    rd = rng.normal(size=(n, 3))
    rd /= np.linalg.norm(rd, axis=1, keepdims=True)
    return ro.astype(np.float32), rd.astype(np.float32)


def test_binary32_triangle_test_matches_fp64_away_from_edges(port):
    nodes, bricks, _ = golden_octree()
    occ = port.occluder_triangles(occluder_surfaces(), 0)
    S = port.scene(nodes, bricks, occ)
    ro, rd = _rays(1500, 4)
    h32 = port.occluded(S, ro, rd)
    h64, margin = port.occluded_fp64(S, ro.astype(np.float64), rd.astype(np.float64))
    far = margin > 1e-5
    assert far.mean() > 0.98
    assert np.array_equal(h32[far], h64[far])
    assert 0.1 < h32.mean() < 0.9  # both answers occur
    # known answers: through a triangle's centroid (hit), the same ray reversed
    # (the triangle is behind: miss unless another one is hit), parallel to a triangle (miss)
    areas = np.linalg.norm(np.cross(occ[:, 4:7], occ[:, 8:11]), axis=1)
    assert (areas == 0).any()  # the sphere's poles: degenerate triangles are never hit
    k = int(np.argmax(areas[:-2]))  # a sphere or small triangle (the ground quad is the last two)
    t = occ[k]
    cen = t[0:3] + (t[4:7] + t[8:11]) / 3
    n = np.cross(t[4:7], t[8:11])
    n /= np.linalg.norm(n)
    o = (cen + 0.3 * n).astype(np.float32)
    d = (-n).astype(np.float32)
    S1 = port.scene(nodes, bricks, np.ascontiguousarray(occ[k:k + 1]))
    assert port.occluded(S1, o[None], d[None])[0] == 1
    assert port.occluded(S1, o[None], (-d)[None])[0] == 0
    e = (t[4:7] / np.linalg.norm(t[4:7])).astype(np.float32)
    assert port.occluded(S1, o[None], e[None])[0] == 0


def test_occluders_act_only_in_the_embree_build(port):
    nodes, bricks, _ = golden_octree()
    occ = port.occluder_triangles(occluder_surfaces(), 0)
    keep = []
    cfg = c0_cfg(32, 32)
    P = port.params(cfg, keep)
    plain = port.render_tile(port.scene(nodes, bricks), P, 0, 0, 32, 32, 8, seed=3)
    with_occ = port.render_tile(port.scene(nodes, bricks, occ), P, 0, 0, 32, 32, 8, seed=3)
    for a, b in zip(plain[:2], with_occ[:2]):
        assert np.array_equal(a, b)
    cfg["embree"] = True
    Pe = port.params(cfg, keep)
    e_plain = port.render_tile(port.scene(nodes, bricks), Pe, 0, 0, 32, 32, 8, seed=3)
    e_occ = port.render_tile(port.scene(nodes, bricks, occ), Pe, 0, 0, 32, 32, 8, seed=3)
    for a, b in zip(plain[:2], e_plain[:2]):
        assert np.array_equal(a, b)  # no occluders, no depth texture: the builds agree
    # the sphere shadows the cloud and the ground blocks light from below:
    # less light, the same alpha (occlusion never changes a path's decisions)
    for a, b in zip(e_plain[:2], e_occ[:2]):
        assert (b[..., :3] <= a[..., :3] + 1e-6).all() and b[..., :3].sum() < 0.97 * a[..., :3].sum()
        assert np.array_equal(a[..., 3], b[..., 3])


def test_embree_build_zeroes_alpha_of_depth_cut(port):
    nodes, bricks, _ = golden_octree()
    S = port.scene(nodes, bricks)
    keep = []
    cfg = c0_cfg(48, 48)
    cfg["depth"] = depth_texture(48, 48)
    cfg["depthcomp"] = True
    a = port.render_tile(S, port.params(cfg, keep), 0, 0, 48, 48, 8, seed=6)
    cfg["embree"] = True
    b = port.render_tile(S, port.params(cfg, keep), 0, 0, 48, 48, 8, seed=6)
    # light is unchanged (a cut path gathers none in either build); alpha drops
    # by the cut samples
    assert np.array_equal(a[0][..., :3], b[0][..., :3]) and np.array_equal(a[1][..., :3], b[1][..., :3])
    assert (b[0][..., 3] <= a[0][..., 3]).all() and b[0][..., 3].sum() < a[0][..., 3].sum()
