"""CPU oracle for the droplet-render volumetric path-tracing hot path.

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py may import this package; the
droplet_b200 product never does.

Two checkers live here:
  * oracle/_ref/libdroplet_ref.so -- the reference's own hot-path sources
    (src/kernel.cpp, KernelOctree.cpp, KernelSampler.cpp, ArHosekSkyModel.cpp)
    compiled unmodified with a TBB stand-in (oracle/Makefile `ref`);
  * oracle/_port/liboracle_port.so -- a C restatement of the same path
    (oracle/port/*.c), which also holds the OpenVDB-free scene build and the
    FP64 quadrature references.
"""
from .oracle import Port, Reference, ref_available, port_available, reference_src  # noqa: F401
