"""droplet_b200: B200 (sm_100a) implementation of droplet-render's volumetric
path-tracing hot path behind a plain C ABI (include/droplet_b200.h).

Modules:
  _native    ctypes binding of libdroplet_b200.so (fails loudly when absent)
  scene      octree + brick build (host, native) and layout
  renderer   RenderKernel equivalent: upload, parameters, tile render, probes
  sky        Hosek-Wilkie dataset parsing and state cook
  camera     view / projection matrices in the reference's conventions
  workloads  seeded synthetic density recipes
"""
from . import _native  # noqa: F401

__all__ = ["_native", "camera", "scene", "renderer", "sky", "workloads"]
