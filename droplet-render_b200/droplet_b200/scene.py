"""Octree + brick scenes: building (native, host) and device upload.

`build_octree` wraps dr_build_octree: the OpenVDB-free part of the
reference's Scene::Initialize (src/scene.cpp:676-762, 840-908), fed with
sparse 8^3 blocks.  The result is the reference's node records
(OctreeStructure, src/scene.h:21-31) and the FOG brick pool.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N

NODE_DTYPE = np.dtype([("ce", "<f4", 4), ("chn", "<u4", 8), ("volx", "<u4", 2), ("qval", "<f4", 2)])
assert NODE_DTYPE.itemsize == 64


@dataclass
class Octree:
    nodes: np.ndarray     # NODE_DTYPE records
    bricks: np.ndarray    # (n_leaves, 512) float32
    mlevel: int
    sdf_bricks: np.ndarray | None = None  # (n_sdf, 512) float32 surface bricks of leaves with volx[0] set

    @property
    def n_nodes(self) -> int:
        return len(self.nodes)

    @property
    def n_leaves(self) -> int:
        return len(self.bricks)

    def leaf_ids(self) -> np.ndarray:
        return np.nonzero(self.nodes["volx"][:, 1] != N.DR_NONE)[0]

    def nbytes(self) -> int:
        return self.nodes.nbytes + self.bricks.nbytes


def build_octree(block_origin: np.ndarray, block_values: np.ndarray, voxel_size: float, maxdepth: int = 12,
                 threads: int = 0) -> Octree:
    org = np.ascontiguousarray(block_origin, np.int32).reshape(-1, 3)
    vals = np.ascontiguousarray(block_values, np.float32).reshape(-1, 512)
    if len(org) != len(vals):
        raise ValueError("block_origin and block_values differ in length")
    oc = N.DrOctree()
    N.check(N.lib().dr_build_octree(org.ctypes.data, vals.ctypes.data, len(org), float(voxel_size), int(maxdepth),
                                    int(threads), C.byref(oc)))
    try:
        nodes = np.frombuffer(C.string_at(oc.nodes, oc.n_nodes * 64), NODE_DTYPE).copy()
        bricks = np.frombuffer(C.string_at(oc.bricks, oc.n_leaves * 512 * 4), np.float32).reshape(-1, 512).copy()
        mlevel = int(oc.mlevel)
    finally:
        N.lib().dr_octree_free(C.byref(oc))
    return Octree(nodes, bricks, mlevel)


def build_from_dense(grid: np.ndarray, voxel_size: float, maxdepth: int = 12, threads: int = 0) -> Octree:
    """Dense grid indexed [x, y, z]; voxel (i, j, k) at world (i, j, k) * voxel_size."""
    from .workloads import dense_to_blocks

    org, vals = dense_to_blocks(grid)
    return build_octree(org, vals, voxel_size, maxdepth, threads)
